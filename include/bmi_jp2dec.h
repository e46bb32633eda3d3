/*
 * bmi_jp2dec.h — the reference's C decoding interface, re-declared for this library.
 *
 * Interface being replaced: decoder/codec/include/bmi_jp2dec.h:39-118 (configuration
 * flags, stru_dec_param, BMI_dec_info / BMI_dec_init / BMI_dec / BMI_dec_thumbnail /
 * BMI_dec_isr / BMI_dec_exit in the SOFTWARE_MULTI_THREAD build).  Return conventions are
 * the reference's: 0 ok / -1 error, and BMI_dec_thumbnail returns a BMI::Status whose
 * success value is PARSING (decoder/codec/src/dec_jp2.cpp:248-270, :400).
 *
 * Semantics here: BMI_dec_info parses the main header into the parameter block and
 * reports pool sizes; BMI_dec_init checks the caller's pools; BMI_dec decodes the whole
 * codestream on the GPU and writes one plane per component into output[c] as
 * DC-shifted, clamped samples after the inverse MCT (R, G, B for colour pictures;
 * uint8 for bit depths <= 8, uint16 above);
 * BMI_dec_thumbnail does the same at 1/2^resolution size.
 */
#ifndef BMI_JP2DEC_H
#define BMI_JP2DEC_H

#include "bmi_decoder.h"

#define MAX_COMPONENT 4
#define MAX_DWT_LEVEL 10

#ifdef __cplusplus
extern "C" {
#endif

enum enum_dec_configuration {
  CONF_BYPASS = 0x00000001,
  CONF_RESET = 0x00000002,
  CONF_TERMALL = 0x00000004,
  CONF_CAUSAL = 0x00000008,
  CONF_PTERM = 0x00000010,
  CONF_SEGSYM = 0x00000020,
  CONF_SOP = 0x00000040,
  CONF_EPH = 0x00000080,
  CONF_DWT97 = 0x00000100,
  CONF_MCT = 0x00000200,
  CONF_QUANT = 0x00000400,
  CONF_JP2FILE = 0x01000000,
  CONF_VIDEO = 0x02000000,
  CONF_VHDLTB = 0x10000000,
  CONF_OPTIM = 0xC0000000
};

typedef struct tag_stru_dec_param {
  void *mempool[2];
  int pool_size[2];

  void *input;
  void *output[MAX_COMPONENT];
  unsigned int in_size;

  int width;
  int height;
  int bitdepth;
  int format;
  int num_components;

  int cb_width;
  int cb_height;
  int prec_width;
  int prec_height;
  int tile_width;
  int tile_height;
  int tile_num;
  int size_opt;

  int layer;
  int dwt_level;
  int roi_shift;
  Jp2_Progression progression;

  int configuration;

  int guard_bit;
  unsigned int quant_step[1 + 3 * MAX_DWT_LEVEL];
} stru_dec_param;

int BMI_dec_info(stru_dec_param *dec_param, int thread_num);
int BMI_dec_init(stru_dec_param *dec_param, int use_j2k_header, int thread_num);
int BMI_dec_isr(stru_dec_param *dec_param, int fpga_irq);
int BMI_dec(stru_dec_param *dec_param, void *output[MAX_COMPONENT], int use_j2k_header);
#ifdef __cplusplus
BMI::Status BMI_dec_thumbnail(stru_dec_param *dec_param, void *output[MAX_COMPONENT], int resolution,
                              int use_j2k_header);
#else
int BMI_dec_thumbnail(stru_dec_param *dec_param, void *output[MAX_COMPONENT], int resolution, int use_j2k_header);
#endif
int BMI_dec_exit(stru_dec_param *dec_param);

#ifdef __cplusplus
}
#endif

#endif
