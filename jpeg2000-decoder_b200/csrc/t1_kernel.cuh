/*
 * t1_kernel.cuh — EBCOT Tier-1 code-block decoder for sm_100a.
 *
 * One warp per code-block.  The warp keeps the block's stripe context words in shared
 * memory and the MQ registers (A, C, t, T, byte position) in registers.
 * The arithmetic decode is inherently serial, so all 32 lanes execute the same scalar
 * decode in lock-step (uniform control flow, broadcast shared-memory reads); the lanes
 * work in parallel where the data allows it: clearing the state, locating the next
 * non-empty stripe column of a pass with a warp ballot, measuring runs of empty columns
 * in the cleanup pass, and the dequantising, coalesced rewrite of the finished block.
 * Blocks are pulled from a device work queue (atomic counter over a host-sorted order,
 * longest blocks first), so CTAs stay resident and uneven blocks balance out.
 *
 * Latency and occupancy measures, none of which changes a decoded bit:
 *   - two kernel forms: the compact one (long queues, throughput) is kept small for the
 *     instruction cache (many resident warps sit in different passes at once): each pass
 *     walks the rows of a stripe column as a bit mask, inlines each of its decisions once,
 *     and bypass (raw) and MQ decisions share the pass code; the unrolled one (batches that
 *     fit about two waves, latency) unrolls the rows and hands the lanes' chunk words and
 *     masks to the serial loop;
 *   - per 32-column chunk the lanes compute each column's row mask and only columns with
 *     work join the serial loop;
 *   - each MQ context slot holds its probability-table entry (Qe, MPS, both successor
 *     states), so a symbol needs one shared-memory load before its decision;
 *   - code bytes are read as aligned 32-bit words with the next word requested early, so
 *     byte fills do not wait on memory;
 *   - in the cleanup pass a run of all-zero columns whose run-length symbols would all
 *     decode as MPS without renormalisation (C >= k*Qe and A - k*Qe >= 0x8000, scaled) is
 *     consumed in one step: A -= k*Qe, C -= k*Qe;
 *   - samples live in the block's own region of the output buffer, not in shared memory:
 *     they are only written while decoding (significance sets sign + 1.5 * 2^p, a
 *     refinement flips bit p and sets the new midpoint bit), so updates go out as
 *     fire-and-forget atomic XORs: in the compact form a stripe column's at its end from
 *     lanes 0..3 in one instruction, in the unrolled form each 32-column chunk's at its end
 *     from the lanes owning the columns (off the serial chain: C2 Tier-1 10.8 -> 7.9 ms),
 *     and the "first refinement?" context test of the reference ((|v| >> p) < 4, true
 *     exactly on a sample's first refinement) reads a per-sample "refined" bit kept in
 *     shared memory.  A 64x64 block then needs 6 KB of shared memory instead of 13-21 KB,
 *     so more blocks are resident per SM;
 *   - bypass refinement bits of a column are taken together and scattered to their rows.
 *
 * Semantics follow the reference block decoder exactly (decoder/codec/src/
 * bmi_block_decoder.cpp:10-853, bmi_mq_decoder.h/.cpp, bmi_t1_macro.h): same context-word
 * layout, same scaled MQ registers and 0xFF/marker handling, same midpoint ("one and a
 * half") reconstruction bits, same MSB-plane rule including its plane-0 -> plane-1 case for
 * 9/7 blocks (:708-711), and the same 5/3 placement shift (dec_t1_comp.cpp:341-366).  Raw
 * (bypass) passes, context reset, per-pass termination and segmentation symbols follow
 * ITU-T T.800 Annex D (the reference asserts on them).
 */
#pragma once
#include <cstdint>

#include "plan.h"



namespace j2k_dev {

// ---- context-word bits (bmi_t1_macro.h:14-73)
constexpr uint32_t NBR_ROW0 = 0x1EF;
constexpr int MU_POS = 20, PI_POS = 21, CHI_POS = 19;
__device__ __forceinline__ uint32_t ROW_SIG(int k) { return 0x10u << (3 * k); }
__device__ __forceinline__ uint32_t ROW_CHI(int k) { return 1u << (CHI_POS + 3 * k); }
__device__ __forceinline__ uint32_t ROW_MU(int k) { return 1u << (MU_POS + 3 * k); }
__device__ __forceinline__ uint32_t ROW_PI(int k) { return 1u << (PI_POS + 3 * k); }
__device__ __forceinline__ uint32_t ROW_NBR(int k) { return NBR_ROW0 << (3 * k); }
constexpr uint32_t MU_ALL = (1u << 20) | (1u << 23) | (1u << 26) | (1u << 29);
constexpr uint32_t PI_ALL = (1u << 21) | (1u << 24) | (1u << 27) | (1u << 30);
constexpr uint32_t CHI_ALL = (1u << 19) | (1u << 22) | (1u << 25) | (1u << 28);

enum { C_SIG = 0, C_RUN = 9, C_SIGN = 10, C_MAG = 15, C_UNI = 18, N_CTX = 19 };

// Read-only tables (constant memory; every lane of a warp reads the same entry):
//   mq[94]   : entry of state s = idx*2 + mps: .x = Qe << 8 (the scaled register unit),
//              .y = (mps << 16) | (state after an MPS << 8) | state after an LPS
//   zc[3][512]: zero-coding context for LL/LH, HL, HH neighbourhoods
//   sc[256]  : (sign context << 1) | xor bit for an 8-bit (sigma, chi) neighbour index
//   rawmr[r][x]: bypass refinement bits: the n = popcount(r) raw bits x (first decoded in
//              bit n-1) placed on the rows set in r, lowest row first
struct T1Tables {
  uint2 mq[96];
  uint8_t zc[3][512];
  uint8_t sc[256];
  uint8_t rawmr[16][16];
};

// MQ decoder registers.  Code bytes are read as aligned 32-bit words: `cur` holds the byte
// at `ap`, and the word after it is requested as soon as `cur` is entered, so the load has
// several fills (dozens of symbols) to complete before its first byte is needed.
struct Mq {
  int32_t A, C;
  int32_t t, T;
  uint32_t ap, aend;  // byte position and segment end, counted from `w`
  const uint32_t *w;  // the segment's first byte rounded down to a 4-byte boundary
  uint32_t cur, nxt;  // the word holding byte ap and the one after it
};

__device__ __forceinline__ int mq_byte(const Mq &m) {
  return m.ap < m.aend ? (int)((m.cur >> ((m.ap & 3) * 8)) & 0xFF) : 0xFF;
}

__device__ __forceinline__ void mq_advance(Mq &m) {
  m.ap++;
  if (!(m.ap & 3)) {
    m.cur = m.nxt;
    m.nxt = __ldg(m.w + (m.ap >> 2) + 1);
  }
}

// FILL_LSBS, bmi_mq_decoder.h:52-73, as selects: after a 0xFF byte the next byte carries 7
// bits, unless it is a marker (> 0x8F), which is not consumed and reads as 0xFF with 8 bits
__device__ __forceinline__ void mq_fill(Mq &m) {
  const int b = mq_byte(m);
  const bool ff = m.T == 0xFF;
  const bool marker = ff && b > 0x8F;
  m.T = marker ? 0xFF : (ff ? b << 1 : b);
  if (!marker) mq_advance(m);
  m.t = (ff && !marker) ? 7 : 8;
  m.C += m.T;
}

// Init, bmi_mq_decoder.cpp:186-219 (the 0xFF 0xFF termination is virtual: bytes at or past
// `end` read as 0xFF).  The word loads may reach up to 9 bytes past the segment; the code
// byte buffer carries 16 bytes of slack after its last segment.
__device__ __forceinline__ void mq_init(Mq &m, const uint8_t *base, uint32_t len) {
  const uint32_t off = (uint32_t)((uintptr_t)base & 3);
  m.w = reinterpret_cast<const uint32_t *>(base - off);
  m.ap = off;
  m.aend = off + len;
  m.cur = __ldg(m.w);
  m.nxt = __ldg(m.w + 1);
  m.T = 0;
  m.C = 0;
  m.t = 0;
  mq_fill(m);
  m.C <<= m.t;
  mq_fill(m);
  m.C <<= 7;
  m.t -= 7;
  m.A = 0x800000;
}

// Shift until A >= 0x800000, filling a byte whenever t reaches 0 (the reference's
// RENORMALIZE_ONCE loop, taken several shifts at a time; at most two fills, as a fill
// after a 0xFF byte is followed by one of 8 bits)
__device__ __forceinline__ void mq_renorm(Mq &m) {
  int n = __clz(m.A) - 8;
  while (m.t < n) {
    m.A <<= m.t;
    m.C <<= m.t;
    n -= m.t;
    mq_fill(m);
  }
  m.A <<= n;
  m.C <<= n;
  m.t -= n;
}

// MQ_DECODE, bmi_mq_decoder.h:86-128, on a context slot holding its table entry.  Both
// renormalising outcomes (conditional exchange after C < Qe; A below 0x8000 after C >= Qe)
// share one table update and one renormalisation.  EARLY (compact kernel form: fewest
// instructions) returns the common outcome first: C >= Qe and A still >= 0x8000 after
// A -= Qe (MPS, no renormalisation); otherwise (unrolled form: shortest dependency chain)
// the outcome is computed before a single branch.
template <bool EARLY>
__device__ __forceinline__ int mq_decode(Mq &m, uint2 *cx, const uint2 *tab) {
  const uint2 e = *cx;
  const int32_t q = (int32_t)e.x;
  m.A -= q;
  const bool ex = m.C < q;
  if constexpr (EARLY) {
    if (!ex && m.A >= 0x800000) {
      m.C -= q;
      return (int)((e.y >> 16) & 1);
    }
    const bool lps = (m.A < q) != ex;
    if (ex) m.A = q;
    else m.C -= q;
    *cx = tab[lps ? (e.y & 0xFF) : ((e.y >> 8) & 0xFF)];
    mq_renorm(m);
    return (int)((e.y >> 16) & 1) ^ (int)lps;
  } else {
    const bool lps = ex ? (m.A >= q) : (m.A < q);
    const int sym = (int)((e.y >> 16) & 1) ^ (int)lps;
    if (!ex) m.C -= q;
    if (ex || m.A < 0x800000) {
      *cx = tab[lps ? (e.y & 0xFF) : ((e.y >> 8) & 0xFF)];
      if (ex) m.A = q;
      mq_renorm(m);
    }
    return sym;
  }
}

// MQ_DECODE_START (fixed Qe 0x5601, MPS 0, no adaptation), bmi_mq_decoder.h:131-169
__device__ __forceinline__ int mq_uniform(Mq &m) {
  int ret = 0;
  if (m.C < 0x560100) {
    if (m.A >= (0x560100 << 1)) ret = 1;
    if (!m.t) mq_fill(m);
    m.C <<= 1;
    m.t--;
    m.A = 0x560100 << 1;
  } else {
    m.A -= 0x560100;
    m.C -= 0x560100;
    if (m.A < 0x800000) {
      if (m.A < 0x560100) ret = 1;
      mq_renorm(m);
    }
  }
  return ret;
}

struct Raw {
  uint32_t pos, end;
  const uint8_t *base;
  uint32_t c;
  int ct, last;
};
__device__ __forceinline__ void raw_init(Raw &r, const uint8_t *base, uint32_t len) {
  r.base = base;
  r.pos = 0;
  r.end = len;
  r.c = 0;
  r.ct = 0;
  r.last = 0;
}
// T.800 D.6: after 0xFF the next byte carries 7 bits; bytes past the end read as 0xFF
__device__ __forceinline__ int raw_bit(Raw &r) {
  if (r.ct == 0) {
    int b = r.pos < r.end ? (int)__ldg(r.base + r.pos) : 0xFF;
    r.pos++;
    r.ct = (r.last == 0xFF) ? 7 : 8;
    r.last = b;
    r.c = (uint32_t)b;
  }
  r.ct--;
  return (int)((r.c >> r.ct) & 1);
}

// ---- samples: raw int32 (bit 31 sign, magnitude with midpoint bit) built in global memory:
// a sample's significance writes its first value (nothing touched it before), refinements
// XOR into it; samples that never become significant are never written while decoding (the
// final rewrite gives them 0 from the significance bits in shared memory), so the block
// region needs no zero-fill.  The lane that writes a sample's first value also issues its
// refinements, so each sample's updates stay in program order.  While a 32-column chunk
// of a stripe is decoded, each column's update goes to the lane that owns the column (one
// select in the serial loop); at the end of the chunk every lane issues its column's row
// updates as fire-and-forget atomics, consecutive lanes on consecutive columns (nothing reads
// the samples while decoding, and XOR updates commute).
struct Samples {
  int32_t *base;      // the block's first sample in the output buffer
  uint32_t stride;    // elements per row
  int lane;
  // column update `upd`: bits 0..3 rows updated, bits 4..7 the sign (significance pass) or
  // the decoded refinement bit (refinement pass) of each row
  // one column's update from lanes 0..3 in one warp instruction, straight from the serial
  // loop (compact form: cheapest when every resident warp competes for issue slots)
  template <bool REFINE>
  __device__ __forceinline__ void apply(int row0, int col, uint32_t upd, int plane) const {
    if (lane < 4 && ((upd >> lane) & 1)) {
      const uint32_t bit = (upd >> (4 + lane)) & 1;
      unsigned int *at = reinterpret_cast<unsigned int *>(base + (size_t)(row0 + lane) * stride + col);
      if (REFINE) atomicXor(at, ((1u - bit) << plane) | ((1u << plane) >> 1));
      else *at = (bit << 31) + (1u << plane) + ((1u << plane) >> 1);  // first value of the sample
    }
  }
  // a chunk's updates, each lane issuing its own column's (unrolled form: the serial loop of
  // a latency-bound batch keeps only a select per column)
  template <bool REFINE>
  __device__ __forceinline__ void flush(int row0, int col, uint32_t upd, int plane) const {
    if (!(upd & 0xF)) return;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!((upd >> k) & 1)) continue;
      const uint32_t bit = (upd >> (4 + k)) & 1;
      unsigned int *at = reinterpret_cast<unsigned int *>(base + (size_t)(row0 + k) * stride + col);
      if (REFINE) atomicXor(at, ((1u - bit) << plane) | ((1u << plane) >> 1));
      else *at = (bit << 31) + (1u << plane) + ((1u << plane) >> 1);  // first value of the sample
    }
  }
};

// per-warp decode state in shared memory
struct BlockSmem {
  uint32_t *cw;  // context words: (stripes + 2) rows of (w + 3) words, + 2
  uint8_t *rf;   // per stripe column: bit k set once row k has been refined
  uint2 *cx;     // 18 MQ context slots (table entries)
  Samples sp;
  int w, gap;
};

__device__ __forceinline__ uint32_t *cword(const BlockSmem &b, int s, int c) {
  return b.cw + (s + 1) * b.gap + 1 + c;
}

// sign context index of row k: bit 0 sigma up, 1 chi up, 2 sigma down, 3 chi down,
// 4 sigma left, 5 chi left, 6 sigma right, 7 chi right
__device__ __forceinline__ int sign_index(uint32_t cw, uint32_t wl, uint32_t wr, int k) {
  uint32_t v = cw >> (3 * k);
  uint32_t chi_up = (k == 0) ? (cw >> 18) & 1 : (v >> 16) & 1;
  uint32_t idx = ((v >> 1) & 1) | (chi_up << 1) | (((v >> 7) & 1) << 2) | (((v >> 22) & 1) << 3);
  uint32_t l = wl >> (3 * k), r = wr >> (3 * k);
  idx |= ((l >> 4) & 1) << 4 | ((l >> 19) & 1) << 5 | ((r >> 4) & 1) << 6 | ((r >> 19) & 1) << 7;
  return (int)idx;
}

// Mark row k of the column at `wp` significant with sign `sym`: spread sigma / chi to the
// neighbouring words (bmi_block_decoder.cpp:53-101 and the row 1..3 variants).  In CAUSAL
// blocks (T.800 D.7) a stripe's last row sees the next stripe as insignificant, so row 0
// spreads nothing upward; the flag sits in a spare byte of the refined-rows array (see
// causal_flag) and is read only here.
__device__ __forceinline__ uint8_t &causal_flag(const BlockSmem &b) { return b.rf[b.gap - 1]; }
__device__ __forceinline__ void spread_sig(const BlockSmem &b, uint32_t *wp, uint32_t &cw, int k, int sym) {
  if (k == 0 && !causal_flag(b)) {
    uint32_t *up = wp - b.gap;
    up[-1] |= 0x100u << 9;
    up[0] |= (0x80u << 9) | ((uint32_t)sym << 31);
    up[1] |= 0x40u << 9;
  } else if (k == 3) {
    uint32_t *dn = wp + b.gap;
    dn[-1] |= 0x04u;
    dn[0] |= 0x02u | ((uint32_t)sym << 18);
    dn[1] |= 0x01u;
  }
  wp[-1] |= 0x20u << (3 * k);
  wp[1] |= 0x08u << (3 * k);
  cw |= ROW_SIG(k) | ((uint32_t)sym << (CHI_POS + 3 * k));
}

enum { P_SIGPROP = 0, P_MAGREF = 1, P_CLEANUP = 2 };

// one decision: a raw bit in a bypass segment, else an MQ symbol
template <bool UNROLLED>
__device__ __forceinline__ int decide(bool israw, Raw &raw, Mq &mq, uint2 *slot, const uint2 *tab) {
  return israw ? raw_bit(raw) : mq_decode<!UNROLLED>(mq, slot, tab);
}

// Sign of row k (raw bit, or MQ symbol in the sign context of its neighbours XOR the
// context's prediction bit), then the sample becomes significant; returns its column update
template <bool UNROLLED>
__device__ __forceinline__ uint32_t significant(const BlockSmem &b, uint32_t *wp, uint32_t &cw, int k, bool israw,
                                                Raw &raw, Mq &mq, const T1Tables &T) {
  int flip = 0, slot = C_SIGN;
  if (!israw) {
    const int sv = T.sc[sign_index(cw, wp[-1], wp[1], k)];
    slot += sv >> 1;
    flip = sv & 1;
  }
  const int sg = decide<UNROLLED>(israw, raw, mq, b.cx + slot, T.mq) ^ flip;
  spread_sig(b, wp, cw, k, sg);
  return (1u << k) | ((uint32_t)sg << (4 + k));  // this row's column update
}

// Rows of a stripe column that pass a pass's test, as a 4-bit mask (bit k = row k), with
// v = word >> 3k holding row k's bits at row 0's positions:
// (v & FORBID) == 0 && (v & NEED) == NEED && (ANY == 0 || (v & ANY) != 0)
template <uint32_t FORBID, uint32_t NEED, uint32_t ANY>
__device__ __forceinline__ uint32_t row_mask(uint32_t cw) {
  uint32_t m = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t v = cw >> (3 * k);
    const bool ok = !(v & FORBID) && (v & NEED) == NEED && (ANY == 0 || (v & ANY) != 0);
    m |= (uint32_t)ok << k;
  }
  return m;
}
constexpr uint32_t V_SIG = 0x10u, V_CHI = 1u << CHI_POS, V_MU = 1u << MU_POS, V_PI = 1u << PI_POS;

// Two forms of each pass's column code, with identical decisions:
//   UNROLLED = false (throughput): the rows to visit are a 4-bit mask walked with ffs, and
//     each decision is inlined once, so the kernel stays small for the instruction cache
//     when many warps are resident and sit in different passes;
//   UNROLLED = true (latency): the four rows are unrolled with constant masks, trading
//     code size for a shorter dependency chain per symbol, for batches too small to fill
//     the GPU, whose time is the serial time of their longest blocks.

// significance propagation of one stripe column (bmi_block_decoder.cpp:10-215): rows
// not yet significant with a significant neighbour; a row that becomes significant can
// make the rows below it eligible
template <bool UNROLLED>
__device__ __forceinline__ uint32_t sigprop_column(const BlockSmem &b, uint32_t *wp, uint32_t &cw, uint32_t todo,
                                                   bool israw, const uint8_t *zc, Raw &raw, Mq &mq,
                                                   const T1Tables &T) {
  uint32_t upd = 0;
  if constexpr (UNROLLED) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t v = cw >> (3 * k);
      if (!(v & NBR_ROW0) || (v & (V_SIG | V_CHI))) continue;
      const int d = decide<UNROLLED>(israw, raw, mq, b.cx + C_SIG + zc[v & NBR_ROW0], T.mq);
      cw |= ROW_PI(k);
      if (d) upd |= significant<UNROLLED>(b, wp, cw, k, israw, raw, mq, T);
    }
  } else {
    while (todo) {
      const int k = __ffs(todo) - 1;
      todo &= todo - 1;
      const int d = decide<UNROLLED>(israw, raw, mq, b.cx + C_SIG + zc[(cw >> (3 * k)) & NBR_ROW0], T.mq);
      cw |= ROW_PI(k);
      if (d) {
        upd |= significant<UNROLLED>(b, wp, cw, k, israw, raw, mq, T);
        todo = row_mask<V_SIG | V_CHI, 0u, NBR_ROW0>(cw) & (0xEu << k);
      }
    }
  }
  return upd;
}

// magnitude refinement of one stripe column (bmi_block_decoder.cpp:217-349): rows
// significant before this bit-plane
template <bool UNROLLED>
__device__ __forceinline__ uint32_t magref_column(const BlockSmem &b, uint32_t cw, uint32_t rows, uint8_t *rf,
                                                  bool israw, Raw &raw, Mq &mq, const T1Tables &T) {
  const uint32_t refined = *rf;
  uint32_t bits = 0;
  if (israw) {
    // bypass: the column's refinement bits are consecutive raw bits, taken together
    const int n = __popc(rows);
    uint32_t x = 0;
    if (raw.ct >= n) {
      x = (raw.c >> (raw.ct - n)) & ((1u << n) - 1u);
      raw.ct -= n;
    } else {
      for (int i = 0; i < n; ++i) x = (x << 1) | (uint32_t)raw_bit(raw);
    }
    if (rows) *rf = (uint8_t)(refined | rows);
    return rows | ((uint32_t)T.rawmr[rows][x] << 4);
  }
#pragma unroll
  for (int i = 0; i < (UNROLLED ? 4 : 1); ++i) {
    uint32_t todo = UNROLLED ? (rows & (1u << i)) : rows;
    while (todo) {
      const int k = UNROLLED ? i : __ffs(todo) - 1;
      todo &= todo - 1;
      // first refinement of this sample <=> (|v| >> p) < 4 in the reference
      const int ctx = C_MAG + (((refined >> k) & 1) ? 2 : (((cw >> (3 * k)) & NBR_ROW0) ? 1 : 0));
      bits |= (uint32_t)decide<UNROLLED>(israw, raw, mq, b.cx + ctx, T.mq) << (4 + k);
    }
  }
  if (rows) *rf = (uint8_t)(refined | rows);
  return rows | bits;  // column update: rows refined and their decoded bits
}

// cleanup of one stripe column (bmi_block_decoder.cpp:351-586): an all-zero column is
// coded in run mode (one run-length symbol; if it is 1, two uniform symbols give the row
// of the first significant sample, whose sign follows directly); then every row not yet
// coded in this bit-plane
template <bool UNROLLED>
__device__ __forceinline__ uint32_t cleanup_column(const BlockSmem &b, uint32_t *wp, uint32_t &cw, uint32_t todo,
                                                   const uint8_t *zc, Raw &raw, Mq &mq, const T1Tables &T) {
  int forced = -1;
  if (cw == 0) {
    // run-length symbol, then the two uniform symbols (the reference's fixed-Qe
    // MQ_DECODE_START is an ordinary decision on a context pinned at state 46)
    int r = 0;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
      const int d = mq_decode<!UNROLLED>(mq, b.cx + (i == 0 ? C_RUN : C_UNI), T.mq);
      if (i == 0 && !d) return 0;  // the whole column stays insignificant
      r = (r << 1) | d;
    }
    forced = r & 3;
    todo = (0xFu << forced) & 0xFu;
  }
  uint32_t upd = 0;
#pragma unroll
  for (int i = 0; i < (UNROLLED ? 4 : 1); ++i) {
    uint32_t rows = UNROLLED ? (todo & (1u << i)) : todo;
    while (rows) {
      const int k = UNROLLED ? i : __ffs(rows) - 1;
      rows &= rows - 1;
      if (k != forced && !mq_decode<!UNROLLED>(mq, b.cx + C_SIG + zc[(cw >> (3 * k)) & NBR_ROW0], T.mq)) continue;
      upd |= significant<UNROLLED>(b, wp, cw, k, false, raw, mq, T);
    }
  }
  return upd;
}

// One coding pass over the block.  Columns are visited in 32-column chunks: a ballot
// selects the columns with work (non-zero word for significance propagation, a refinable
// sample for refinement, every column for cleanup); a sample that becomes significant makes
// the next column non-zero, so that column joins the set.  In cleanup, a run of all-zero
// columns whose run-length symbols would all decode as MPS without renormalisation
// (C >= k*Qe and A - k*Qe >= 0x8000, scaled) is consumed in one step: A -= k*Qe, C -= k*Qe.
// Each pass inlines its decision sites once, without unrolling over the four rows, so the
// kernel stays small enough for the instruction cache when many warps are resident.
// PASS (P_SIGPROP / P_MAGREF / P_CLEANUP) and RAW (a bypass segment: raw bits instead of MQ
// symbols) are compile-time constants, so each instantiation carries only its own pass's
// column code and no decision tests either flag at run time.
template <bool UNROLLED, int PASS, bool RAW>
__device__ __forceinline__ void run_pass(const BlockSmem &b, int stripes, int p, const uint8_t *zc, Mq &mq, Raw &raw,
                                         const T1Tables &T, int lane) {
  constexpr int pass = PASS;
  constexpr bool israw = RAW;
  for (int s = 0; s < stripes; ++s) {
    uint32_t *row = cword(b, s, 0);
    uint8_t *rrow = b.rf + s * b.gap;
    for (int c0 = 0; c0 < b.w; c0 += 32) {
      __syncwarp();
      // lane-parallel view of the chunk: each lane's word and the rows its pass would
      // visit; only columns with work join the serial loop (a column reached from the left
      // by a new significant sample joins it then).  The unrolled form also hands the
      // lanes' words and masks to the serial loop: a column's word changes only when its
      // left neighbour gains a significant sample (`dirty`), so only those are reloaded.
      // The compact form keeps fewer values live across the serial loop (registers bound
      // its occupancy) and reloads each word.
      constexpr bool LP = UNROLLED;
      const int c = c0 + lane;
      const bool valid = c < b.w;
      const uint32_t word = valid ? row[c] : 0u;
      uint32_t mask;
      bool work;
      if (pass == P_SIGPROP) {
        mask = row_mask<V_SIG | V_CHI, 0u, NBR_ROW0>(word);
        work = mask != 0;
      } else if (pass == P_MAGREF) {
        mask = row_mask<0u, V_SIG | V_MU, 0u>(word);
        work = mask != 0;
      } else {
        mask = row_mask<V_SIG | V_CHI | V_PI, 0u, 0u>(word);
        work = word == 0 || mask != 0;  // run mode, or rows not yet coded in this bit-plane
      }
      uint32_t live = __ballot_sync(0xffffffffu, valid && work);
      uint32_t zero = __ballot_sync(0xffffffffu, valid && word == 0);
      uint32_t dirty = 0;
      uint32_t my_upd = 0;  // this lane's column update, flushed at the end of the chunk
      // compact form: the lanes' cleanup / refinement masks go through shared memory (they
      // depend on a column's own rows only, so they hold while the chunk is decoded; a
      // register copy would raise the register count above the occupancy budget)
      uint8_t *lane_masks = reinterpret_cast<uint8_t *>(b.cx + N_CTX);
      if (!LP && pass != P_SIGPROP) {
        lane_masks[lane] = (uint8_t)mask;
        __syncwarp();
      }
      while (live) {
        const int bit = __ffs(live) - 1;
        if (pass == P_CLEANUP && ((zero >> bit) & 1)) {
          const uint2 e = b.cx[C_RUN];
          const int32_t q = (int32_t)e.x;
          const int32_t m = min(mq.A - 0x800000, mq.C);
          if (!((e.y >> 16) & 1) && m >= q) {
            int n = __clz(__brev(~(zero >> bit)));  // zero columns from `bit` on, in this chunk
            if (n * q > m) n = m / q;
            mq.A -= n * q;
            mq.C -= n * q;
            const uint32_t span = n >= 32 ? 0xffffffffu : ((1u << n) - 1u);
            live &= ~(span << bit);
            continue;
          }
        }
        live &= live - 1;
        const int col = c0 + bit;
        uint32_t *wp = row + col;
        uint32_t cw, lane_word = 0, lane_mask = 0;
        bool dty = true;
        if (LP) {
          lane_word = __shfl_sync(0xffffffffu, word, bit);
          lane_mask = __shfl_sync(0xffffffffu, mask, bit);
          dty = (dirty >> bit) & 1;
          cw = dty ? *wp : lane_word;
        } else {
          cw = *wp;
        }
        if (pass == P_MAGREF) {
          const uint32_t rows = LP ? lane_mask : lane_masks[bit];
          const uint32_t upd = magref_column<UNROLLED>(b, cw, rows, rrow + col, israw, raw, mq, T);
          if constexpr (UNROLLED) my_upd = lane == bit ? upd : my_upd;
          else b.sp.apply<true>(4 * s, col, upd, p);
          continue;
        }
        uint32_t upd;
        if (pass == P_SIGPROP) {
          const uint32_t todo = dty ? row_mask<V_SIG | V_CHI, 0u, NBR_ROW0>(cw) : lane_mask;
          upd = sigprop_column<UNROLLED>(b, wp, cw, todo, israw, zc, raw, mq, T);
        } else {
          // own-row bits do not change from the left, so the lane's mask holds; a column
          // that was all-zero may have been reached from the left and is not any more
          const uint32_t todo = LP ? ((dty && lane_word == 0) ? row_mask<V_SIG | V_CHI | V_PI, 0u, 0u>(cw) : lane_mask)
                                   : lane_masks[bit];
          upd = cleanup_column<UNROLLED>(b, wp, cw, todo, zc, raw, mq, T);
        }
        *wp = cw;
        const bool newsig = (upd & 0xF) != 0;
        if constexpr (UNROLLED) my_upd = lane == bit ? upd : my_upd;
        else if (newsig) b.sp.apply<false>(4 * s, col, upd, p);
        if (newsig && bit < 31) {
          if (pass == P_SIGPROP) live |= 1u << (bit + 1);
          zero &= ~(1u << (bit + 1));
          if (LP) dirty |= 1u << (bit + 1);
        }
      }
      if constexpr (UNROLLED) b.sp.flush<pass == P_MAGREF>(4 * s, c, my_upd, p);
      if (pass == P_CLEANUP) {
        // end of the bit-plane for this chunk's columns: mu |= sigma, pi cleared
        // (bmi_block_decoder.cpp:571-573); no later decision of this pass reads a column's
        // own mu / pi bits
        __syncwarp();
        if (valid) {
          uint32_t w = row[c];
          w |= (w << (MU_POS - 4)) & MU_ALL;
          row[c] = w & ~PI_ALL;
        }
      }
    }
  }
  __syncwarp();
}

__device__ __forceinline__ void init_states(uint2 *cx, const uint2 *tab) {
  // bmi_mq_decoder.cpp:65-79: (state 0, MPS 0) except sig ctx 0 -> state 4, run -> state 3
  for (int i = 0; i < N_CTX; ++i) cx[i] = tab[0];
  cx[C_SIG] = tab[4 << 1];
  cx[C_RUN] = tab[3 << 1];
  cx[C_UNI] = tab[46 << 1];
}

__device__ __forceinline__ bool seg_starts(int flags, int j) {
  if (j == 0) return true;
  if (flags & J2K_CB_TERMALL) return true;
  int type = (j - 1) % 3;
  return (flags & J2K_CB_BYPASS) && j >= 10 && type != 1;
}

// MSB plane and pass count of a block (bmi_block_decoder.cpp:603-622, :708-711)
__device__ __forceinline__ void block_planes(const j2k_cblk &cb, int &bit_plane, int &num_passes) {
  const int missing = cb.missing;
  const int p_max = 30 - missing;
  num_passes = 3 * p_max - 2;
  if (num_passes > cb.num_passes) num_passes = cb.num_passes;
  if (cb.flags & J2K_CB_IRREV) {
    bit_plane = (int)cb.mb - 1 - missing;
  } else {
    if (((int)cb.mb - missing) * 3 - 2 <= 0) num_passes = 0;
    bit_plane = -1 - missing;
  }
  if (bit_plane < 0) bit_plane = p_max;
  if (bit_plane == 0) bit_plane = 1;
}

// Decode one code-block with the whole warp.  Returns a status (0 ok).
template <bool UNROLLED>
__device__ __forceinline__ int decode_block(const j2k_cblk &cb, const uint8_t *__restrict__ bytes, const uint32_t *__restrict__ seglens,
                            const BlockSmem &b, const T1Tables &T, int lane, int bit_plane, int num_passes) {
  const int w = cb.w, h = cb.h;
  const int stripes = (h + 3) >> 2;
  // clear the context words and refinement bits (the samples need no clearing: see
  // Samples); mark OOB columns and a partial last stripe
  const int nwords = (stripes + 2) * b.gap + 2;
  for (int i = lane; i < nwords; i += 32) b.cw[i] = 0;
  for (int i = lane; i < stripes * b.gap; i += 32) b.rf[i] = 0;
  __syncwarp();
  const uint32_t oob = CHI_ALL;
  for (int s = lane; s < stripes; s += 32) {
    uint32_t *r = cword(b, s, w);
    r[0] = oob;
    r[1] = oob;
    r[2] = oob;
  }
  if (h & 3) {
    uint32_t m = (h & 3) == 1 ? (ROW_CHI(1) | ROW_CHI(2) | ROW_CHI(3))
                              : ((h & 3) == 2 ? (ROW_CHI(2) | ROW_CHI(3)) : ROW_CHI(3));
    for (int c = lane; c < w; c += 32) *cword(b, stripes - 1, c) = m;
  }
  if (lane == 0) {
    init_states(b.cx, T.mq);
    // stripe 0's refined-rows row has three unused bytes past the last column
    causal_flag(b) = (cb.flags & J2K_CB_CAUSAL) ? 1 : 0;
  }
  __syncwarp();
  if (num_passes > 0 && 30 - (int)cb.missing <= 0) return 1;

  const int multi = (cb.flags & (J2K_CB_BYPASS | J2K_CB_TERMALL)) != 0;
  const uint8_t *zc = T.zc[cb.band == 3 ? 2 : (cb.band == 1 ? 1 : 0)];
  const uint8_t *data = bytes + cb.data_off;
  Mq mq;
  Raw raw;
  mq.A = mq.C = mq.t = mq.T = 0;
  mq.ap = mq.aend = mq.cur = mq.nxt = 0;
  mq.w = reinterpret_cast<const uint32_t *>(bytes);
  raw_init(raw, data, 0);
  uint32_t seg_pos = 0;
  int seg_idx = 0;
  bool israw = false;
  int status = 0;
  for (int k = 0, type = 2; k < num_passes; ++k, ++type) {
    if (type == 3) {
      type = 0;
      bit_plane--;
    }
    if (bit_plane < 0) {
      status = 2;
      break;
    }
    if (seg_starts(multi ? cb.flags : 0, k)) {
      uint32_t len;
      if (multi) {
        if (seg_idx >= cb.nseg) {
          status = 3;
          break;
        }
        len = __ldg(seglens + cb.seg_off + seg_idx);
        seg_idx++;
      } else {
        len = cb.data_len;
      }
      if (seg_pos + len > cb.data_len) {
        status = 4;
        break;
      }
      israw = (cb.flags & J2K_CB_BYPASS) && k >= 10 && type != 2;
      if (israw) raw_init(raw, data + seg_pos, len);
      else mq_init(mq, data + seg_pos, len);
      seg_pos += len;
    }
    if (type == P_CLEANUP) run_pass<UNROLLED, P_CLEANUP, false>(b, stripes, bit_plane, zc, mq, raw, T, lane);
    else if (type == P_SIGPROP && israw) run_pass<UNROLLED, P_SIGPROP, true>(b, stripes, bit_plane, zc, mq, raw, T, lane);
    else if (type == P_SIGPROP) run_pass<UNROLLED, P_SIGPROP, false>(b, stripes, bit_plane, zc, mq, raw, T, lane);
    else if (israw) run_pass<UNROLLED, P_MAGREF, true>(b, stripes, bit_plane, zc, mq, raw, T, lane);
    else run_pass<UNROLLED, P_MAGREF, false>(b, stripes, bit_plane, zc, mq, raw, T, lane);
    if (type == 2 && (cb.flags & J2K_CB_SEGSYM))
      for (int i = 0; i < 4; ++i) mq_uniform(mq);
    if (cb.flags & J2K_CB_RESET) {
      __syncwarp();
      if (lane == 0) init_states(b.cx, T.mq);
      __syncwarp();
    }
  }
  __syncwarp();
  return status;
}

}  // namespace j2k_dev
