/*
 * j2k_oracle.h — CPU restatement of the reference decoder's hot path (test infrastructure
 * only; see j2k_oracle.c for the file:line map into the reference).
 */
#ifndef J2K_ORACLE_H
#define J2K_ORACLE_H

#include <stdint.h>

#include "../jpeg2000-decoder_b200/csrc/plan.h"

#ifdef __cplusplus
extern "C" {
#endif

/* OutputFormat values of the reference (decoder/common/include/codec_datatype.h:38-51) */
enum {
  ORACLE_FMT_32BITS_ARGB = 0,
  ORACLE_FMT_48BITS_RGB = 1,
  ORACLE_FMT_24BITS_RGB = 2,
  ORACLE_FMT_32BITS_4COMPONENTS = 3,
  ORACLE_FMT_64BITS_4COMPONENTS = 4,
  ORACLE_FMT_48BITS_3COMPONENTS = 5,
  ORACLE_FMT_24BITS_3COMPONENTS = 6,
  ORACLE_FMT_64BITS_ARGB = 8
};

/* Tier-1 of one code-block: w*h int32 samples in the reference's raw form
 * (bit 31 sign, magnitude with midpoint bits).  Returns 0 or an error status. */
int oracle_t1_block(const j2k_cblk *cb, const uint8_t *bytes, const uint32_t *seglens, int32_t *out);
/* Tier-1 decisions (MQ symbols incl. run-length and uniform ones, raw bits) decoded so far
 * by this process: a workload statistic for the benchmark report. */
unsigned long long oracle_decisions(void);
/* Tier-1 of all blocks placed into the coefficient buffer (int32 for 5/3, float for 9/7). */
int oracle_t1_place(const j2k_cblk *cblks, int ncb, const uint8_t *bytes, const uint32_t *seglens, void *coef,
                    int32_t *status);
/* In-place inverse DWT of one tile-component region. */
int oracle_idwt(const j2k_tilecomp *tc, int reversible, int ref_compat, void *coef_base);
/* Inverse MCT + DC shift + clamp + pack of all tiles. */
int oracle_output(const j2k_image_info *info, const j2k_tilecomp *tcs, int ntc, const void *coef, int fmt,
                  uint8_t *out, int pitch_px);
int oracle_format_bytes(int fmt);
/* Whole decode: returns 0 or the number of code-blocks with a Tier-1 error. */
int oracle_decode(const j2k_image_info *info, const j2k_cblk *cblks, int ncb, const uint8_t *bytes,
                  const uint32_t *seglens, const j2k_tilecomp *tcs, int ntc, int ref_compat, int fmt, uint8_t *out,
                  void *coef_out);

#ifdef __cplusplus
}
#endif
#endif
