/*
 * plan.h — flat, device-ready description of one decoded image ("decode plan").
 *
 * The host front end (codestream.cpp: markers, tiles, Tier-2 packet headers) turns a
 * codestream into these arrays; the CUDA kernels and the CPU oracle both consume them.
 * It replaces the reference's per-code-block pass lists (stru_code_block / stru_coding_pass,
 * decoder/codec/include/dec_stru.h:194-277) and the per-subband stripe geometry kept by
 * CudaManager / CpuDwtDecoder::InitPicture (decoder/codec/src/bmi_cpu_dwt_decoder.cpp:851-1120).
 *
 * Coefficient layout in HBM: one region per tile-component, row-major with the
 * tile-component width as stride, subbands in Mallat order (LL_L top-left; for every
 * resolution r the HL band right of, the LH band below and the HH band diagonal to the
 * resolution r-1 image).  Tier-1 writes each code-block straight into its band position;
 * the inverse DWT then rebuilds every resolution inside the same footprint.
 */
#ifndef J2K_PLAN_H
#define J2K_PLAN_H

#include <stdint.h>

#define J2K_MAX_LEVELS 10
#define J2K_MAX_COMPONENTS 4

/* code-block flags */
enum {
  J2K_CB_BYPASS = 0x01,  /* T.800 selective arithmetic coding bypass */
  J2K_CB_RESET = 0x02,   /* context reset after every pass */
  J2K_CB_TERMALL = 0x04, /* every pass terminated */
  J2K_CB_CAUSAL = 0x08,  /* vertically stripe-causal contexts */
  J2K_CB_PTERM = 0x10,
  J2K_CB_SEGSYM = 0x20,  /* segmentation symbol after each cleanup pass */
  J2K_CB_IRREV = 0x40,   /* 9/7 path: output float = coefficient * gain */
  J2K_CB_HI_ONLY = 0x80  /* reserved */
};

/* One Tier-1 work item (40 bytes). */
typedef struct j2k_cblk {
  uint32_t data_off;   /* offset of this block's coded bytes in the batch byte buffer */
  uint32_t data_len;   /* total coded bytes, all segments and layers concatenated */
  uint64_t out_off;    /* element offset of the block's top-left sample in the coefficient buffer */
  uint32_t out_stride; /* elements per row of the tile-component region */
  uint32_t seg_off;    /* first entry of this block's segment lengths in the segment table */
  float gain;          /* 9/7: Delta' * K_h * K_v (reference gain folding); 5/3: unused */
  uint16_t w, h;       /* block size in samples */
  uint8_t num_passes;  /* coding passes included over all layers */
  uint8_t missing;     /* zero (missing) most significant bit-planes */
  uint8_t band;        /* 0 LL, 1 HL, 2 LH, 3 HH */
  uint8_t mb;          /* magnitude bit-planes M_b = exponent + guard bits - 1 (T.800 E.1.1.1; the
                          reference's "numbps" for one guard bit) */
  uint8_t flags;       /* J2K_CB_* */
  uint8_t nseg;        /* codeword segments (>= 1 when num_passes > 0) */
  uint16_t spqcd;      /* raw QCD/QCC step value of the band (exponent << 11 | mantissa, or exponent) */
} j2k_cblk;

/* One tile-component: the inverse DWT/MCT work for one region of the coefficient buffer. */
typedef struct j2k_tilecomp {
  uint64_t coef_off;   /* element offset of the region */
  int32_t x0, y0;      /* tile-component origin on its component's grid at the output resolution,
                          relative to the component's origin (j2k_image_info comp_x0 / comp_y0) */
  int32_t w, h;        /* tile-component size */
  int32_t levels;      /* decomposition levels of this tile-component */
  int32_t comp, tile;
  int32_t res_w[J2K_MAX_LEVELS + 1], res_h[J2K_MAX_LEVELS + 1]; /* resolution r = 0..levels */
} j2k_tilecomp;

typedef struct j2k_image_info {
  int32_t width, height, ncomp, bitdepth;
  int32_t is_signed;
  int32_t tile_w, tile_h, ntiles_x, ntiles_y;
  int32_t levels;        /* COD levels (main header) */
  int32_t reversible;    /* 1: 5/3, 0: 9/7 */
  int32_t mct;           /* COD multiple component transform flag */
  int32_t layers, progression, cbw, cbh, cbstyle, guard_bits;
  int32_t num_cblks, num_tilecomps, num_segs;
  uint64_t coded_bytes;  /* Tier-1 bytes in the plan */
  uint64_t coef_elems;   /* elements of the coefficient buffer */
  /* component sampling (SIZ XRsiz / YRsiz) and each component's own grid at the output
   * resolution: absolute origin and size.  A tile-component's (x0, y0) are relative to its
   * component's origin.  Picture pixel (X, Y) (relative to the picture origin
   * origin_x, origin_y) shows component c's sample floor((origin_x + X) / sub_x[c]) -
   * comp_x0[c] (likewise in y): sub-sampled components are replicated. */
  int32_t origin_x, origin_y;
  int32_t sub_x[J2K_MAX_COMPONENTS], sub_y[J2K_MAX_COMPONENTS];
  int32_t comp_x0[J2K_MAX_COMPONENTS], comp_y0[J2K_MAX_COMPONENTS];
  int32_t comp_w[J2K_MAX_COMPONENTS], comp_h[J2K_MAX_COMPONENTS];
} j2k_image_info;

#endif
