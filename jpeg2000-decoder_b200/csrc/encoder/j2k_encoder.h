/*
 * j2k_encoder.h — minimal JPEG 2000 Part-1 (ITU-T T.800) codestream writer.
 *
 * The reference library ships an empty encoder shell (decoder/core/src/encoderconcrete.cpp),
 * so every codestream the tests and the benchmark decode is produced here from seeded
 * synthetic images.  Supported: reversible 5/3 + RCT, irreversible 9/7 + ICT with
 * scalar-expounded quantisation, rectangular tiles anchored at the origin, 32/64 code-blocks,
 * quality layers chosen by slope thresholds, LRCP/RLCP/RPCL/PCRL/CPRL progression with one
 * precinct per resolution, progression volumes (POC, main or tile-part header), tile-parts
 * (optionally interleaved across tiles), SOP / EPH markers, packed packet headers (PPM or
 * PPT), the BYPASS / RESET / TERMALL / CAUSAL / SEGSYM mode switches, and sub-sampled
 * components (XRsiz / YRsiz, e.g. YCbCr 4:2:0 and 4:2:2).
 *
 * The irreversible path writes one guard bit by default: the reference's Tier-1 places the
 * most significant magnitude bit at (expn - 1 - missing) (decoder/codec/src/
 * bmi_block_decoder.cpp:708-710), which is only the T.800 position when G == 1.
 */
#ifndef J2K_ENCODER_H
#define J2K_ENCODER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum j2kenc_progression { J2KENC_LRCP = 0, J2KENC_RLCP = 1, J2KENC_RPCL = 2, J2KENC_PCRL = 3, J2KENC_CPRL = 4 };

/* code-block style bits, as written in the COD marker (T.800 Table A.19) */
enum j2kenc_mode {
  J2KENC_BYPASS = 0x01,
  J2KENC_RESET = 0x02,
  J2KENC_TERMALL = 0x04,
  J2KENC_CAUSAL = 0x08, /* vertically stripe-causal contexts */
  J2KENC_PTERM = 0x10,  /* accepted, termination is the plain T.800 flush */
  J2KENC_SEGSYM = 0x20
};

/* marker options (T.800 A.6.1 Scod, A.7.4-A.7.5, A.8) */
enum j2kenc_marker { J2KENC_SOP = 1, J2KENC_EPH = 2, J2KENC_PPM = 4, J2KENC_PPT = 8 };

typedef struct j2kenc_params {
  int reversible;     /* 1: 5/3 integer + RCT; 0: 9/7 + ICT */
  int levels;         /* decomposition levels, 0..10 */
  int cbw_exp;        /* log2 code-block width  (2..10, cbw_exp + cbh_exp <= 12) */
  int cbh_exp;        /* log2 code-block height */
  int tile_w;         /* 0: one tile covering the image */
  int tile_h;
  int num_layers;     /* 1..32 */
  double layer_bpp[32]; /* cumulative target bits per pixel for each layer; <= 0: all passes */
  int progression;    /* j2kenc_progression */
  int mode;           /* OR of j2kenc_mode */
  int use_mct;        /* apply RCT/ICT when there are >= 3 components */
  int guard_bits;     /* 0: 1 for 9/7, 2 for 5/3 */
  double base_step;   /* 9/7: quantiser step for a unit-energy band, in sample units */
  int num_threads;    /* 0: hardware concurrency */
  int markers;        /* OR of j2kenc_marker (PPM and PPT exclude each other) */
  int tile_parts;     /* tile-parts per tile, packets split evenly (0 or 1: one) */
  int interleave_tile_parts; /* write part k of every tile before part k + 1 */
  int num_poc;        /* progression volumes (0: the COD progression); they must cover every packet */
  int poc[8][6];      /* per volume: first resolution, first component, layer end, resolution end,
                         component end, progression */
  int poc_in_tiles;   /* 0: POC in the main header; 1: in the first tile-part header of each tile */
  int sub_x[4], sub_y[4]; /* component sub-sampling XRsiz / YRsiz (0 or 1: none).  Component c keeps
                             the samples of its plane at reference-grid points (i * sub_x, j * sub_y);
                             the tile size over each factor must be a multiple of 2^levels, and
                             the MCT needs the first three components sampled alike */
} j2kenc_params;

void j2kenc_default_params(j2kenc_params *p);

/*
 * Encode an image of `ncomp` planes (plane-major, row-major, `bitdepth`-bit unsigned samples
 * in uint16) into a raw J2K codestream.  *out is allocated with malloc; free it with
 * j2kenc_free.  Returns 0 on success, a negative value on a parameter error.
 */
int j2kenc_encode(const uint16_t *planes, int width, int height, int ncomp, int bitdepth,
                  const j2kenc_params *params, uint8_t **out, size_t *out_len);
void j2kenc_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
