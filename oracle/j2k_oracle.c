/*
 * j2k_oracle.c — CPU restatement of the reference decoder's hot path.  TEST
 * INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load this library as the checker; the product never links or calls it.
 *
 * What it restates (xxjjss/jpeg2000-decoder, paths relative to the project root):
 *   - MQ decoder, scaled-register form (A, C pre-shifted by 8; FILL_LSBS with the 0xFF /
 *     >0x8F marker rule; forced 0xFF 0xFF termination): decoder/codec/src/bmi_mq_decoder.h:52-169,
 *     bmi_mq_decoder.cpp:33-79 (tables, initial states), :186-258 (Init/Decode/DecodeInit).
 *   - Tier-1 block decoding with Kakadu-style stripe context words (sigma 3x6 neighbourhood,
 *     chi/mu/pi bits): bmi_t1_macro.h:14-73, bmi_block_decoder.cpp:10-215 (significance
 *     propagation), :217-349 (magnitude refinement), :351-586 (cleanup + run mode),
 *     :589-853 (block driver: MSB plane, pass count, one codeword segment, midpoint bits).
 *     The zero-word skipping of the reference is an equivalent speed-up and is not restated.
 *   - Placement into the subband buffer: dec_t1_comp.cpp:283-426 (9/7 raw sign-magnitude;
 *     5/3 ">> (31 - numbps)").
 *   - Dequantisation and gain folding: bmi_cpu_dwt_decoder.cpp:1035-1044, :1433-1473,
 *     FETCHPIXEL_INT at :2287.
 *   - Inverse 9/7 lifting (delta, gamma, beta, alpha with D = S - c*(L+R) in float):
 *     :2283-2485 (rows), :2766-3310 and vdwt_analyst_line :4975-4993 (columns).
 *   - Inverse 5/3 lifting: :2609-2659 (rows), :3311-3534 (columns, including the
 *     bottom-edge behaviour reproduced when ref_compat is set).
 *   - Inverse ICT / RCT, DC shift, clamp, LIFT and packing: :3570-3841, :3936-4130,
 *     :4133-4598.
 * Extensions beyond the reference (it asserts on them, bmi_mq_decoder.cpp:206-210): raw
 * (bypass) passes, context RESET, per-pass termination and segmentation symbols, restated
 * from ITU-T T.800 Annex D.
 */
#include "j2k_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- MQ decoder -------- */
/* T.800 Table C.2; the reference builds the same transitions, bmi_mq_decoder.cpp:37-62 */
static const uint16_t QE[47] = {0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801,
                                0x3001, 0x2401, 0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401,
                                0x3001, 0x2801, 0x2401, 0x2201, 0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101,
                                0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1, 0x0221, 0x0141, 0x0111, 0x0085,
                                0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
static const uint8_t NMPS[47] = {1,  2,  3,  4,  5,  38, 7,  8,  9,  10, 11, 12, 13, 29, 15, 16,
                                 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32,
                                 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 45, 46};
static const uint8_t NLPS[47] = {1,  6,  9,  12, 29, 33, 6,  14, 14, 14, 17, 18, 20, 21, 14, 14,
                                 15, 16, 17, 18, 19, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29,
                                 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 46};

typedef struct {
  uint8_t idx, mps;
} ctx_t;

typedef struct {
  int32_t A, C, t, T;
  const uint8_t *p, *end; /* bytes at or after `end` read as 0xFF */
} mq_t;

static int rd(const mq_t *m) { return m->p < m->end ? *m->p : 0xFF; }

static void mq_fill(mq_t *m) {
  if (m->T == 0xFF) {
    if (rd(m) > 0x8F) {
      m->t = 8; /* marker: synthesise 1s, do not advance */
    } else {
      m->T = rd(m) << 1;
      m->p++;
      m->t = 7;
    }
  } else {
    m->T = rd(m);
    m->p++;
    m->t = 8;
  }
  m->C += m->T;
}

static void mq_init(mq_t *m, const uint8_t *buf, uint32_t len) {
  m->p = buf;
  m->end = buf + len; /* the reference writes 0xFF 0xFF at buf[len] (bmi_mq_decoder.cpp:195) */
  m->T = 0;
  m->C = 0;
  m->t = 0;
  mq_fill(m);
  m->C <<= m->t;
  mq_fill(m);
  m->C <<= 7;
  m->t -= 7;
  m->A = 0x800000;
}

static void mq_renorm_once(mq_t *m) {
  if (!m->t) mq_fill(m);
  m->A <<= 1;
  m->C <<= 1;
  m->t--;
}

/* Decisions decoded (MQ symbols and raw bits), counted per thread and added to a process
 * total at the end of each block: a workload statistic for the benchmark report. */
static _Thread_local unsigned long long t_decisions;
static unsigned long long g_decisions;

static int mq_decode(mq_t *m, ctx_t *cx) {
  t_decisions++;
  int32_t q = (int32_t)QE[cx->idx] << 8;
  int ret = cx->mps;
  int sw = (QE[cx->idx] == 0x5601 && NLPS[cx->idx] != 46);
  m->A -= q;
  if (m->C < q) {
    if (m->A < q) {
      cx->idx = NMPS[cx->idx];
    } else {
      ret ^= 1;
      if (sw) cx->mps ^= 1;
      cx->idx = NLPS[cx->idx];
    }
    m->A = q;
    do mq_renorm_once(m);
    while (m->A < 0x800000);
  } else {
    m->C -= q;
    if (m->A < 0x800000) {
      if (m->A < q) {
        ret ^= 1;
        if (sw) cx->mps ^= 1;
        cx->idx = NLPS[cx->idx];
      } else {
        cx->idx = NMPS[cx->idx];
      }
      do mq_renorm_once(m);
      while (m->A < 0x800000);
    }
  }
  return ret;
}

/* fixed-probability (Qe 0x5601, MPS 0) symbol: bmi_mq_decoder.h:131-169 (MQ_DECODE_START) */
static int mq_decode_uniform(mq_t *m) {
  t_decisions++;
  int ret = 0;
  if (m->C < 0x560100) {
    if (m->A >= (0x560100 << 1)) ret = 1;
    if (!m->t) mq_fill(m);
    m->C <<= 1;
    m->t--;
    m->A = 0x560100 << 1;
  } else {
    m->A -= 0x560100;
    m->C -= 0x560100;
    if (m->A < 0x800000) {
      if (m->A < 0x560100) {
        ret = 1;
        do mq_renorm_once(m);
        while (m->A < 0x800000);
      } else {
        mq_renorm_once(m);
      }
    }
  }
  return ret;
}

/* raw (bypass) bits, T.800 D.6: after a 0xFF byte the next byte carries 7 bits */
typedef struct {
  const uint8_t *p, *end;
  uint32_t c;
  int ct, last;
} raw_t;

static void raw_init(raw_t *r, const uint8_t *buf, uint32_t len) {
  r->p = buf;
  r->end = buf + len;
  r->c = 0;
  r->ct = 0;
  r->last = 0;
}
static int raw_bit(raw_t *r) {
  t_decisions++;
  if (r->ct == 0) {
    int b = r->p < r->end ? *r->p : 0xFF;
    r->p++;
    r->ct = (r->last == 0xFF) ? 7 : 8;
    r->last = b;
    r->c = (uint32_t)b;
  }
  r->ct--;
  return (r->c >> r->ct) & 1;
}

/* ------------------------------------------------------------ context words ---------- */
/* bit layout of one stripe-column word (bmi_t1_macro.h:14-73) */
#define S_TL 0x01
#define S_TC 0x02
#define S_TR 0x04
#define S_CL 0x08
#define S_SELF 0x10
#define S_CR 0x20
#define S_BL 0x40
#define S_BC 0x80
#define S_BR 0x100
#define NBR_ROW0 0x1EF
#define MU_POS 20
#define PI_POS 21
#define CHI_POS 19
#define CHI_PREV (1u << 18)
#define CHI_NEXT (1u << 31)
#define ROW_CHI(k) (1u << (CHI_POS + 3 * (k)))
#define ROW_MU(k) (1u << (MU_POS + 3 * (k)))
#define ROW_PI(k) (1u << (PI_POS + 3 * (k)))
#define ROW_SIG(k) ((uint32_t)S_SELF << (3 * (k)))
#define ROW_NBR(k) ((uint32_t)NBR_ROW0 << (3 * (k)))

enum { C_SIG = 0, C_RUN = 9, C_SIGN = 10, C_MAG = 15, N_CTX = 18 };

static void init_contexts(ctx_t *s) {
  /* bmi_mq_decoder.cpp:65-79: all states 0 except sig-prop ctx 0 -> 4 and run -> 3 */
  for (int i = 0; i < N_CTX; ++i) {
    s[i].idx = 0;
    s[i].mps = 0;
  }
  s[C_SIG].idx = 4;
  s[C_RUN].idx = 3;
}

/* zero-coding context of a 9-bit neighbourhood (TL,TC,TR,CL,x,CR,BL,BC,BR = bits 0..8),
 * T.800 Table D.1; the reference keeps these as lut_ctx_lllh / _hl / _hh (dec_t1.h:10-113) */
static int zc_context(uint32_t nb, int band) {
  int h = ((nb >> 3) & 1) + ((nb >> 5) & 1);
  int v = ((nb >> 1) & 1) + ((nb >> 7) & 1);
  int d = (nb & 1) + ((nb >> 2) & 1) + ((nb >> 6) & 1) + ((nb >> 8) & 1);
  if (band == 3) {
    int hv = h + v;
    if (d >= 3) return 8;
    if (d == 2) return hv >= 1 ? 7 : 6;
    if (d == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
    return hv >= 2 ? 2 : hv;
  }
  if (band == 1) {
    int t = h;
    h = v;
    v = t;
  }
  if (h == 2) return 8;
  if (h == 1) return v >= 1 ? 7 : (d >= 1 ? 6 : 5);
  if (v == 2) return 4;
  if (v == 1) return 3;
  return d >= 2 ? 2 : d;
}

/* sign context (T.800 Table D.3) from the four neighbours' (sigma, chi) pairs; the
 * reference packs the same eight bits into lut_ctx_sign / lut_ctx_xor (dec_t1.h:179-237) */
static void sign_context(int sl, int xl, int sr, int xr, int su, int xu, int sd, int xd, int *ctx, int *flip) {
  int H = (sl ? (xl ? -1 : 1) : 0) + (sr ? (xr ? -1 : 1) : 0);
  int V = (su ? (xu ? -1 : 1) : 0) + (sd ? (xd ? -1 : 1) : 0);
  if (H > 1) H = 1;
  if (H < -1) H = -1;
  if (V > 1) V = 1;
  if (V < -1) V = -1;
  int x = 0;
  if (H < 0 || (H == 0 && V < 0)) {
    H = -H;
    V = -V;
    x = 1;
  }
  *flip = x;
  if (H == 1) *ctx = V == 1 ? 4 : (V == 0 ? 3 : 2);
  else *ctx = V == 1 ? 1 : 0;
}

typedef struct {
  uint32_t *cw;    /* context words, rows of (w + 3), one guard row above and below */
  int32_t *sp;     /* samples, (stripes * 4) x w */
  int w, h, stripes, gap;
  int band;
  int causal; /* CAUSAL mode switch (T.800 D.7): a stripe's last row sees the next stripe as
                 insignificant, so a row-0 sample spreads nothing upward */
} blk_t;

static inline uint32_t *word(blk_t *b, int stripe, int col) { return b->cw + (size_t)(stripe + 1) * b->gap + 1 + col; }

/* decode the sign of row k of the column whose word is `w0` and mark it significant */
static int decode_sign(blk_t *b, int s, int c, int k, mq_t *mq, ctx_t *st, raw_t *raw) {
  uint32_t *wp = word(b, s, c);
  uint32_t cw = *wp;
  int sym;
  if (raw) {
    sym = raw_bit(raw);
  } else {
    int su, xu, sd, xd;
    if (k == 0) {
      su = (cw >> 1) & 1; /* S_TC: row -1 centre */
      xu = (cw & CHI_PREV) ? 1 : 0;
    } else {
      su = (cw & ROW_SIG(k - 1)) ? 1 : 0;
      xu = (cw & ROW_CHI(k - 1)) ? 1 : 0;
    }
    if (k == 3) {
      sd = (cw >> 16) & 1; /* row 4 centre */
      xd = (cw & CHI_NEXT) ? 1 : 0;
    } else {
      sd = (cw & ROW_SIG(k + 1)) ? 1 : 0;
      xd = (cw & ROW_CHI(k + 1)) ? 1 : 0;
    }
    uint32_t wl = wp[-1], wr = wp[1];
    int sl = (wl & ROW_SIG(k)) ? 1 : 0, xl = (wl & ROW_CHI(k)) ? 1 : 0;
    int sr = (wr & ROW_SIG(k)) ? 1 : 0, xr = (wr & ROW_CHI(k)) ? 1 : 0;
    int ctx, flip;
    sign_context(sl, xl, sr, xr, su, xu, sd, xd, &ctx, &flip);
    sym = mq_decode(mq, &st[C_SIGN + ctx]) ^ flip;
  }
  /* propagate sigma / chi (bmi_block_decoder.cpp:87-96, :128-130, :158-160, :190-198) */
  if (k == 0 && !b->causal) {
    uint32_t *up = wp - b->gap;
    up[-1] |= S_BR << 9;
    up[0] |= (S_BC << 9) | ((uint32_t)sym << 31);
    up[1] |= S_BL << 9;
  }
  if (k == 3) {
    uint32_t *dn = wp + b->gap;
    dn[-1] |= S_TR;
    dn[0] |= S_TC | ((uint32_t)sym << 18);
    dn[1] |= S_TL;
  }
  wp[-1] |= (uint32_t)S_CR << (3 * k);
  wp[1] |= (uint32_t)S_CL << (3 * k);
  *wp |= ROW_SIG(k) | ((uint32_t)sym << (CHI_POS + 3 * k));
  return sym;
}

static void pass_sigprop(blk_t *b, int p, mq_t *mq, ctx_t *st, raw_t *raw) {
  int32_t one_and_half = (1 << p) + ((1 << p) >> 1);
  for (int s = 0; s < b->stripes; ++s)
    for (int c = 0; c < b->w; ++c) {
      uint32_t *wp = word(b, s, c);
      for (int k = 0; k < 4; ++k) {
        uint32_t cw = *wp;
        if (!(cw & ROW_NBR(k)) || (cw & (ROW_SIG(k) | ROW_CHI(k)))) continue;
        int sym = raw ? raw_bit(raw) : mq_decode(mq, &st[C_SIG + zc_context((cw >> (3 * k)) & NBR_ROW0, b->band)]);
        if (!sym) {
          *wp |= ROW_PI(k);
        } else {
          int sg = decode_sign(b, s, c, k, mq, st, raw);
          *wp |= ROW_PI(k);
          b->sp[(size_t)(4 * s + k) * b->w + c] = (int32_t)(((uint32_t)sg << 31) + (uint32_t)one_and_half);
        }
      }
    }
}

static void pass_magref(blk_t *b, int p, mq_t *mq, ctx_t *st, raw_t *raw) {
  int32_t half = (1 << p) >> 1;
  for (int s = 0; s < b->stripes; ++s)
    for (int c = 0; c < b->w; ++c) {
      uint32_t cw = *word(b, s, c);
      for (int k = 0; k < 4; ++k) {
        if ((cw & (ROW_MU(k) | ROW_SIG(k))) != (ROW_MU(k) | ROW_SIG(k))) continue;
        int32_t *v = &b->sp[(size_t)(4 * s + k) * b->w + c];
        int32_t val = *v;
        int sym;
        if (raw) {
          sym = raw_bit(raw);
        } else {
          int32_t mag = (val & 0x7FFFFFFF) >> p;
          int ctx = C_MAG;
          if (mag < 4) {
            if (cw & ROW_NBR(k)) ctx++;
          } else {
            ctx += 2;
          }
          sym = mq_decode(mq, &st[ctx]);
        }
        val ^= (int32_t)((uint32_t)(1 - sym) << p);
        val |= half;
        *v = val;
      }
    }
}

static void pass_cleanup(blk_t *b, int p, mq_t *mq, ctx_t *st) {
  int32_t one_and_half = (1 << p) + ((1 << p) >> 1);
  for (int s = 0; s < b->stripes; ++s)
    for (int c = 0; c < b->w; ++c) {
      uint32_t *wp = word(b, s, c);
      int k0 = 0;
      if (*wp == 0) {
        /* run mode (bmi_block_decoder.cpp:376-404) */
        if (!mq_decode(mq, &st[C_RUN])) continue;
        int r = mq_decode_uniform(mq);
        r = (r << 1) | mq_decode_uniform(mq);
        int sg = decode_sign(b, s, c, r, mq, st, NULL);
        b->sp[(size_t)(4 * s + r) * b->w + c] = (int32_t)(((uint32_t)sg << 31) + (uint32_t)one_and_half);
        k0 = r + 1;
      }
      for (int k = k0; k < 4; ++k) {
        uint32_t cw = *wp;
        if (cw & (ROW_SIG(k) | ROW_CHI(k) | ROW_PI(k))) continue;
        int sym = mq_decode(mq, &st[C_SIG + zc_context((cw >> (3 * k)) & NBR_ROW0, b->band)]);
        if (sym) {
          int sg = decode_sign(b, s, c, k, mq, st, NULL);
          b->sp[(size_t)(4 * s + k) * b->w + c] = (int32_t)(((uint32_t)sg << 31) + (uint32_t)one_and_half);
        }
      }
      /* mu |= sigma, pi cleared (bmi_block_decoder.cpp:571-573) */
      uint32_t cw = *wp;
      cw |= (cw << (MU_POS - 4)) & (ROW_MU(0) | ROW_MU(1) | ROW_MU(2) | ROW_MU(3));
      cw &= ~(ROW_PI(0) | ROW_PI(1) | ROW_PI(2) | ROW_PI(3));
      *wp = cw;
    }
}

static int seg_starts(int flags, int j) {
  int type = (j == 0) ? 2 : (j - 1) % 3;
  if (j == 0) return 1;
  if (flags & J2K_CB_TERMALL) return 1;
  return (flags & J2K_CB_BYPASS) && j >= 10 && type != 1;
}

unsigned long long oracle_decisions(void) { return __atomic_load_n(&g_decisions, __ATOMIC_RELAXED); }

static int t1_block(const j2k_cblk *cb, const uint8_t *bytes, const uint32_t *seglens, int32_t *out);

int oracle_t1_block(const j2k_cblk *cb, const uint8_t *bytes, const uint32_t *seglens, int32_t *out) {
  t_decisions = 0;
  const int rc = t1_block(cb, bytes, seglens, out);
  __atomic_fetch_add(&g_decisions, t_decisions, __ATOMIC_RELAXED);
  return rc;
}

static int t1_block(const j2k_cblk *cb, const uint8_t *bytes, const uint32_t *seglens, int32_t *out) {
  const int w = cb->w, h = cb->h;
  const int stripes = (h + 3) >> 2;
  const int irrev = (cb->flags & J2K_CB_IRREV) != 0;
  int32_t *sp = (int32_t *)calloc((size_t)stripes * 4 * w, sizeof(int32_t));
  const int gap = w + 3;
  uint32_t *cwbuf = (uint32_t *)calloc((size_t)(stripes + 2) * gap + 2, sizeof(uint32_t));
  int status = 0;
  memset(out, 0, sizeof(int32_t) * (size_t)w * h);
  if (!sp || !cwbuf) {
    free(sp);
    free(cwbuf);
    return -2;
  }
  blk_t b = {cwbuf, sp, w, h, stripes, gap, cb->band, (cb->flags & J2K_CB_CAUSAL) != 0};
  /* OOB words after every stripe row and a partial last stripe (bmi_block_decoder.cpp:616-705) */
  const uint32_t oob = ROW_CHI(0) | ROW_CHI(1) | ROW_CHI(2) | ROW_CHI(3);
  for (int s = 0; s < stripes; ++s) {
    uint32_t *r = word(&b, s, w);
    r[0] = r[1] = r[2] = oob;
  }
  if (h & 3) {
    uint32_t m = (h & 3) == 1 ? (ROW_CHI(1) | ROW_CHI(2) | ROW_CHI(3)) : (h & 3) == 2 ? (ROW_CHI(2) | ROW_CHI(3)) : ROW_CHI(3);
    for (int c = 0; c < w; ++c) *word(&b, stripes - 1, c) = m;
  }
  int npass_cb = cb->num_passes;
  int missing = cb->missing;
  /* pass count and MSB plane (bmi_block_decoder.cpp:603-622, :708-711) */
  int p_max = 30 - missing;
  int num_passes = 3 * p_max - 2;
  if (num_passes > npass_cb) num_passes = npass_cb;
  int bit_plane;
  if (irrev) {
    bit_plane = (int)cb->mb - 1 - missing;
  } else {
    int maxorig = ((int)cb->mb - missing) * 3 - 2;
    if (maxorig <= 0) num_passes = 0;
    bit_plane = -1 - missing;
  }
  if (bit_plane < 0) bit_plane = p_max;
  if (bit_plane == 0) bit_plane = 1;
  if (num_passes > 0 && p_max <= 0) status = 1;

  ctx_t st[N_CTX];
  init_contexts(st);
  mq_t mq;
  raw_t raw;
  const int multi = (cb->flags & (J2K_CB_BYPASS | J2K_CB_TERMALL)) != 0;
  uint32_t seg_pos = 0;
  int seg_idx = 0;
  int israw = 0;
  for (int k = 0, type = 2; k < num_passes && !status; ++k, ++type) {
    if (type == 3) {
      type = 0;
      bit_plane--;
    }
    if (bit_plane < 0) {
      status = 2;
      break;
    }
    if (seg_starts(multi ? cb->flags : 0, k)) {
      uint32_t len;
      if (multi) {
        if (seg_idx >= cb->nseg) {
          status = 3;
          break;
        }
        len = seglens[cb->seg_off + seg_idx];
        seg_idx++;
      } else {
        len = cb->data_len; /* one segment: every pass of every layer (:735-768) */
      }
      if (seg_pos + len > cb->data_len) {
        status = 4;
        break;
      }
      israw = (cb->flags & J2K_CB_BYPASS) && k >= 10 && type != 2;
      if (israw)
        raw_init(&raw, bytes + cb->data_off + seg_pos, len);
      else
        mq_init(&mq, bytes + cb->data_off + seg_pos, len);
      seg_pos += len;
    }
    if (type == 0)
      pass_sigprop(&b, bit_plane, &mq, st, israw ? &raw : NULL);
    else if (type == 1)
      pass_magref(&b, bit_plane, &mq, st, israw ? &raw : NULL);
    else {
      pass_cleanup(&b, bit_plane, &mq, st);
      if (cb->flags & J2K_CB_SEGSYM) {
        for (int i = 0; i < 4; ++i) mq_decode_uniform(&mq);
      }
    }
    if (cb->flags & J2K_CB_RESET) init_contexts(st);
  }
  for (int y = 0; y < h; ++y) memcpy(out + (size_t)y * w, sp + (size_t)y * w, sizeof(int32_t) * w);
  free(sp);
  free(cwbuf);
  return status;
}

/* dec_t1_comp.cpp:341-366 */
static inline int32_t place53(int32_t v, int numbps) {
  int sh = 31 - numbps;
  if (sh < 0) sh = 0;
  if (sh > 31) sh = 31;
  return v < 0 ? -(int32_t)((uint32_t)(v & 0x7FFFFFFF) >> sh) : (int32_t)((uint32_t)v >> sh);
}
/* FETCHPIXEL_INT, bmi_cpu_dwt_decoder.cpp:2287 */
static inline int32_t signmag_to_int(int32_t v) { return (v & 0x80000000) ? ((v - 1) ^ 0x7FFFFFFF) : (v & 0x7FFFFFFF); }

int oracle_t1_place(const j2k_cblk *cblks, int ncb, const uint8_t *bytes, const uint32_t *seglens, void *coef,
                    int32_t *status) {
  int bad = 0;
  int32_t *tmp = (int32_t *)malloc(sizeof(int32_t) * 4096 * 16);
  if (!tmp) return -2;
  for (int i = 0; i < ncb; ++i) {
    const j2k_cblk *cb = &cblks[i];
    int st = 0;
    if ((size_t)cb->w * cb->h > 4096 * 16) {
      st = 5;
    } else {
      st = oracle_t1_block(cb, bytes, seglens, tmp);
    }
    if (status) status[i] = st;
    if (st) bad++;
    for (int y = 0; y < cb->h; ++y)
      for (int x = 0; x < cb->w; ++x) {
        int32_t v = tmp[(size_t)y * cb->w + x];
        size_t o = cb->out_off + (size_t)y * cb->out_stride + x;
        if (cb->flags & J2K_CB_IRREV) {
          volatile float f = (float)signmag_to_int(v);
          ((float *)coef)[o] = f * cb->gain;
        } else {
          ((int32_t *)coef)[o] = place53(v, cb->mb);
        }
      }
  }
  free(tmp);
  return bad;
}

/* ---------------------------------------------------------------- inverse DWT -------- */
#define K_ALPHA (-1.58613434205992f)
#define K_BETA (-0.05298011857296f)
#define K_GAMMA (0.88291107553093f)
#define K_DELTA (0.44350685204397f)
#define K_LO (1.23017410558578f)

/* one lifting update D = S - c * (L + R), each operation rounded to float */
static inline float lift(float s, float c, float l, float r) {
  volatile float sum = l + r;
  volatile float prod = c * sum;
  volatile float d = s - prod;
  return d;
}

/* inverse 9/7 on one line of n interleaved samples (even origin, whole-sample symmetric) */
static void line97(float *x, int n) {
  if (n < 2) return;
  /* x[-1] = x[1], x[n] = x[n-2] */
#define XM(i) x[(i) < 0 ? -(i) : ((i) >= n ? 2 * (n - 1) - (i) : (i))]
  for (int i = 0; i < n; i += 2) x[i] = lift(x[i], K_DELTA, XM(i - 1), XM(i + 1));
  for (int i = 1; i < n; i += 2) x[i] = lift(x[i], K_GAMMA, XM(i - 1), XM(i + 1));
  for (int i = 0; i < n; i += 2) x[i] = lift(x[i], K_BETA, XM(i - 1), XM(i + 1));
  for (int i = 1; i < n; i += 2) x[i] = lift(x[i], K_ALPHA, XM(i - 1), XM(i + 1));
#undef XM
}

/* inverse 5/3 on one line of interleaved samples (bmi_cpu_dwt_decoder.cpp:2609-2659) */
static void line53(int32_t *x, int n) {
  if (n < 2) return;
#define XM(i) x[(i) < 0 ? -(i) : ((i) >= n ? 2 * (n - 1) - (i) : (i))]
  for (int i = 0; i < n; i += 2) x[i] = x[i] - ((XM(i - 1) + XM(i + 1) + 2) >> 2);
  for (int i = 1; i < n; i += 2) x[i] = x[i] + ((XM(i - 1) + XM(i + 1)) >> 1);
#undef XM
}

/* The reference's VDWT_R53_LINES end-of-column handling (bmi_cpu_dwt_decoder.cpp:3364-3398):
 * recompute the last rows of a column from the low (L) and high (H) inputs as the
 * reference does.  x holds the standard result; L/H are the de-interleaved inputs. */
static void col53_refcompat(int32_t *x, int n, const int32_t *L, const int32_t *H) {
  if (n < 3) return; /* n == 2 is correct in the reference; n == 1 reads outside the column */
  if (!(n & 1)) {
    int m = n / 2;
    x[n - 1] = H[m - 2] + x[n - 2];
  } else {
    int m = (n + 1) / 2;
    int32_t hh = (m >= 3) ? H[m - 3] : H[0];
    int32_t ll = L[m - 2];
    x[n - 1] = ll - ((hh + 1) >> 1);
    x[n - 2] = hh + ((x[n - 1] + x[n - 3]) >> 1);
  }
}

int oracle_idwt(const j2k_tilecomp *tc, int reversible, int ref_compat, void *coef_base) {
  const int W = tc->w;
  int L = tc->levels;
  int maxdim = tc->w > tc->h ? tc->w : tc->h;
  void *line = malloc(sizeof(float) * (size_t)(maxdim + 4));
  void *lo = malloc(sizeof(float) * (size_t)(maxdim + 4));
  void *hi = malloc(sizeof(float) * (size_t)(maxdim + 4));
  if (!line || !lo || !hi) {
    free(line);
    free(lo);
    free(hi);
    return -2;
  }
  const float llg = K_LO * K_LO; /* reconstructed LL gain of the next level (:1599, :1626) */
  for (int r = 1; r <= L; ++r) {
    int rw = tc->res_w[r], rh = tc->res_h[r];
    int lw = tc->res_w[r - 1], lh = tc->res_h[r - 1];
    if (rw <= 0 || rh <= 0) continue;
    if (reversible) {
      int32_t *c = (int32_t *)coef_base + tc->coef_off;
      int32_t *ln = (int32_t *)line;
      /* rows: de-interleave L | H into even / odd positions */
      for (int y = 0; y < rh; ++y) {
        int32_t *row = c + (size_t)y * W;
        for (int x = 0; x < rw; ++x) ln[x] = (x & 1) ? row[lw + x / 2] : row[x / 2];
        line53(ln, rw);
        memcpy(row, ln, sizeof(int32_t) * rw);
      }
      /* columns */
      int32_t *Lc = (int32_t *)lo, *Hc = (int32_t *)hi;
      for (int x = 0; x < rw; ++x) {
        for (int y = 0; y < lh; ++y) Lc[y] = c[(size_t)y * W + x];
        for (int y = 0; y < rh - lh; ++y) Hc[y] = c[(size_t)(lh + y) * W + x];
        for (int y = 0; y < rh; ++y) ln[y] = (y & 1) ? Hc[y / 2] : Lc[y / 2];
        line53(ln, rh);
        if (ref_compat) col53_refcompat(ln, rh, Lc, Hc);
        for (int y = 0; y < rh; ++y) c[(size_t)y * W + x] = ln[y];
      }
    } else {
      float *c = (float *)coef_base + tc->coef_off;
      float *ln = (float *)line;
      for (int y = 0; y < rh; ++y) {
        float *row = c + (size_t)y * W;
        for (int x = 0; x < rw; ++x) {
          if (x & 1) {
            ln[x] = row[lw + x / 2];
          } else {
            float v = row[x / 2];
            if (r > 1 && y < lh) { /* only the reconstructed LL, not the LH band */
              volatile float g = v * llg;
              v = g;
            }
            ln[x] = v;
          }
        }
        line97(ln, rw);
        memcpy(row, ln, sizeof(float) * rw);
      }
      float *Lc = (float *)lo, *Hc = (float *)hi;
      for (int x = 0; x < rw; ++x) {
        for (int y = 0; y < lh; ++y) Lc[y] = c[(size_t)y * W + x];
        for (int y = 0; y < rh - lh; ++y) Hc[y] = c[(size_t)(lh + y) * W + x];
        for (int y = 0; y < rh; ++y) ln[y] = (y & 1) ? Hc[y / 2] : Lc[y / 2];
        line97(ln, rh);
        for (int y = 0; y < rh; ++y) c[(size_t)y * W + x] = ln[y];
      }
    }
  }
  /* a tile-component with zero levels: the 9/7 LL samples carry their full gain already */
  free(line);
  free(lo);
  free(hi);
  return 0;
}

/* ------------------------------------------------------------------ output ------------ */
int oracle_format_bytes(int fmt) {
  switch (fmt) {
    case ORACLE_FMT_32BITS_ARGB: return 4;
    case ORACLE_FMT_48BITS_RGB: return 6;
    case ORACLE_FMT_24BITS_RGB: return 3;
    case ORACLE_FMT_32BITS_4COMPONENTS: return 4;
    case ORACLE_FMT_64BITS_4COMPONENTS: return 8;
    case ORACLE_FMT_48BITS_3COMPONENTS: return 6;
    case ORACLE_FMT_24BITS_3COMPONENTS: return 3;
    case ORACLE_FMT_64BITS_ARGB: return 8;
    default: return 0;
  }
}

static inline int lift_depth(int v, int in, int out) { return in >= out ? v >> (in - out) : v << (out - in); }

static void put_px(uint8_t *px, int fmt, int c, int v) {
  /* memory order of the reference pixel structs: comp with the highest index first
   * (ARGB_32BITS = B,G,R,A = comp3,comp2,comp1,comp0; RGB_24BITS = B,G,R = comp2,comp1,comp0) */
  switch (fmt) {
    case ORACLE_FMT_24BITS_RGB:
    case ORACLE_FMT_24BITS_3COMPONENTS: px[2 - c] = (uint8_t)v; break;
    case ORACLE_FMT_48BITS_RGB:
    case ORACLE_FMT_48BITS_3COMPONENTS: ((uint16_t *)px)[2 - c] = (uint16_t)v; break;
    case ORACLE_FMT_32BITS_ARGB:
    case ORACLE_FMT_32BITS_4COMPONENTS: px[3 - c] = (uint8_t)v; break;
    case ORACLE_FMT_64BITS_ARGB:
    case ORACLE_FMT_64BITS_4COMPONENTS: ((uint16_t *)px)[3 - c] = (uint16_t)v; break;
  }
}

int oracle_output(const j2k_image_info *info, const j2k_tilecomp *tcs, int ntc, const void *coef, int fmt,
                  uint8_t *out, int pitch_px) {
  const int B = info->bitdepth;
  const int pxb = oracle_format_bytes(fmt);
  if (!pxb) return -1;
  const int outdepth = (pxb == 3 || pxb == 4) ? 8 : 16;
  const int rgb = (fmt == ORACLE_FMT_24BITS_RGB || fmt == ORACLE_FMT_48BITS_RGB || fmt == ORACLE_FMT_32BITS_ARGB ||
                   fmt == ORACLE_FMT_64BITS_ARGB);
  const int maxv = (1 << B) - 1, dc = 1 << (B - 1);
  /* group tile-components by tile */
  for (int i = 0; i < ntc; ++i) {
    if (tcs[i].comp != 0) continue;
    const j2k_tilecomp *t0 = &tcs[i];
    const j2k_tilecomp *tc3[4] = {t0, NULL, NULL, NULL};
    int nc = 1;
    for (int j = 0; j < ntc; ++j)
      if (tcs[j].tile == t0->tile && tcs[j].comp > 0 && tcs[j].comp < 4) {
        tc3[tcs[j].comp] = &tcs[j];
        if (tcs[j].comp + 1 > nc) nc = tcs[j].comp + 1;
      }
    const int do_mct = rgb && nc >= 3 && info->mct && tc3[1] && tc3[2];
    /* R, G, B land in bytes 2, 1, 0 of both RGB_24BITS and ARGB_32BITS (alpha = 0) */
    const int slot0 = (pxb == 4 || pxb == 8) ? 1 : 0;
    for (int y = 0; y < t0->h; ++y)
      for (int x = 0; x < t0->w; ++x) {
        uint8_t *px = out + ((size_t)(t0->y0 + y) * pitch_px + (t0->x0 + x)) * pxb;
        memset(px, 0, pxb);
        size_t o = (size_t)y * t0->w + x;
        if (do_mct) {
          if (info->reversible) {
            const int32_t *c0 = (const int32_t *)coef + t0->coef_off, *c1 = (const int32_t *)coef + tc3[1]->coef_off,
                          *c2 = (const int32_t *)coef + tc3[2]->coef_off;
            /* RRct_53, bmi_cpu_dwt_decoder.cpp:3951-3986 */
            int g = c0[o] - ((c1[o] + c2[o]) >> 2) + dc;
            int rr = c2[o] + g, bb = c1[o] + g;
            rr = rr < 0 ? 0 : (rr > maxv ? maxv : rr);
            g = g < 0 ? 0 : (g > maxv ? maxv : g);
            bb = bb < 0 ? 0 : (bb > maxv ? maxv : bb);
            put_px(px, fmt, 0 + slot0, lift_depth(rr, B, outdepth));
            put_px(px, fmt, 1 + slot0, lift_depth(g, B, outdepth));
            put_px(px, fmt, 2 + slot0, lift_depth(bb, B, outdepth));
          } else {
            const float *c0 = (const float *)coef + t0->coef_off, *c1 = (const float *)coef + tc3[1]->coef_off,
                        *c2 = (const float *)coef + tc3[2]->coef_off;
            /* RICT_97_FLOAT, bmi_cpu_dwt_decoder.cpp:3570-3643 */
            const float r_cr = (float)(1.402), g_cb = (float)(-0.34413), g_cr = (float)(-0.71414), b_cb = (float)(1.772);
            volatile float t, u;
            float sh = (float)dc;
            int v[3];
            t = r_cr * c2[o];
            t = c0[o] + t;
            t = t + sh;
            v[0] = (int)(t < 0 ? 0.f : (t > (float)maxv ? (float)maxv : t));
            t = g_cb * c1[o];
            t = c0[o] + t;
            u = g_cr * c2[o];
            t = t + u;
            t = t + sh;
            v[1] = (int)(t < 0 ? 0.f : (t > (float)maxv ? (float)maxv : t));
            t = b_cb * c1[o];
            t = c0[o] + t;
            t = t + sh;
            v[2] = (int)(t < 0 ? 0.f : (t > (float)maxv ? (float)maxv : t));
            for (int k = 0; k < 3; ++k) put_px(px, fmt, k + slot0, lift_depth(v[k], B, outdepth));
          }
        } else {
          /* MergeComponents, bmi_cpu_dwt_decoder.cpp:4283-4370: value of component c into
           * slot c (a single component lands in slot 0: the alpha / last byte) */
          for (int c = 0; c < nc && c < 4; ++c) {
            if (!tc3[c]) continue;
            int v;
            size_t oc = (size_t)y * tc3[c]->w + x;
            if (info->sub_x[c] > 1 || info->sub_y[c] > 1) {
              /* a sub-sampled component shows its nearest-left sample (replication): the
               * sample at floor(absolute pixel / XRsiz) of the component's grid */
              int i = (info->origin_x + t0->x0 + x) / info->sub_x[c] - (info->comp_x0[c] + tc3[c]->x0);
              int j = (info->origin_y + t0->y0 + y) / info->sub_y[c] - (info->comp_y0[c] + tc3[c]->y0);
              i = i < 0 ? 0 : (i >= tc3[c]->w ? tc3[c]->w - 1 : i);
              j = j < 0 ? 0 : (j >= tc3[c]->h ? tc3[c]->h - 1 : j);
              oc = (size_t)j * tc3[c]->w + i;
            }
            if (info->reversible) v = ((const int32_t *)coef)[tc3[c]->coef_off + oc];
            else v = (int)((const float *)coef)[tc3[c]->coef_off + oc];
            v += dc;
            v = v < 0 ? 0 : (v > maxv ? maxv : v);
            if ((pxb == 3 || pxb == 6) && c > 2) continue;
            put_px(px, fmt, c, lift_depth(v, B, outdepth));
          }
        }
      }
  }
  return 0;
}

int oracle_decode(const j2k_image_info *info, const j2k_cblk *cblks, int ncb, const uint8_t *bytes,
                  const uint32_t *seglens, const j2k_tilecomp *tcs, int ntc, int ref_compat, int fmt, uint8_t *out,
                  void *coef_out) {
  void *coef = coef_out;
  int own = 0;
  if (!coef) {
    coef = calloc((size_t)info->coef_elems ? (size_t)info->coef_elems : 1, 4);
    own = 1;
  } else {
    memset(coef, 0, (size_t)info->coef_elems * 4);
  }
  if (!coef) return -2;
  int bad = oracle_t1_place(cblks, ncb, bytes, seglens, coef, NULL);
  for (int i = 0; i < ntc; ++i) oracle_idwt(&tcs[i], info->reversible, ref_compat, coef);
  int rc = 0;
  if (out) rc = oracle_output(info, tcs, ntc, coef, fmt, out, info->width);
  if (own) free(coef);
  return rc ? rc : bad;
}
