/*
 * t1_lanes.cuh — EBCOT Tier-1 with one code-block per lane (t1_form 3, on request only).
 *
 * The warp-per-block kernels (t1_kernel.cuh) run one serial MQ chain per warp, so 31 of
 * every 32 lanes repeat the same scalar work.  Here every lane decodes its own code-block,
 * so that one warp instruction could advance 32 blocks.  Measured on B200 it does not: on
 * 16 1080p 9/7 frames it takes 32.0 ms against the compact warp form's 7.6 ms.  The lanes'
 * pass walks diverge (4.4 of 32 threads active per warp instruction), a decision costs
 * ~200 thread instructions of state-machine bookkeeping, and the 96 blocks' state fills
 * shared memory at one warp per scheduler (issue active 18 %).  It stays as an explicit form,
 * bit-exact, for comparison.  A lane's block state is kept as bit-planes in
 * shared memory, interleaved by lane (element e of lane L at e * 32 + L, so every access
 * of the warp is bank-conflict free whatever position each lane is at):
 *   sig[c], chi[c], pi[c], rho[c]  (c < 64): column bitmaps, bit r = row r of the block:
 *       significance, sign, "coded in this plane's significance pass" and "refined before";
 *   nb[s]  (s < 16): columns of stripe s whose 3-column x 6-row neighbourhood holds a
 *       significant sample (the significance pass's candidate columns, and the cleanup
 *       pass's run-mode test: a full stripe column with nb clear is coded in run mode);
 *   sc[s]  (s < 16): columns of stripe s holding a significant sample (refinement);
 *   cx[19]: the MQ context words: Qe << 8 | MPS << 23 | state << 24.
 * 2380 bytes per 64x64 block, 74.4 KB per warp: three warps per SM, 96 blocks in flight.
 * The lane walks its pass as a small state machine (which decision is pending: zero coding,
 * sign, refinement, run length, run position, segmentation symbol); each step makes one MQ
 * decision and moves to the next pending one, carrying the current stripe column and its
 * two neighbours (6-row windows of sig / chi) in registers.
 *
 * Samples are built in the block's region of the coefficient buffer exactly as in the
 * warp kernels: significance stores sign + 1.5 * 2^p, a refinement XORs bit p and the next
 * midpoint bit; never-significant samples are never written, the final (cooperative,
 * coalesced) rewrite gives them 0 from sig.
 *
 * Blocks up to 64x64 without BYPASS (raw) segments; the warp kernels take the rest.
 * Decisions follow the reference block decoder (decoder/codec/src/bmi_block_decoder.cpp:
 * 10-853, bmi_mq_decoder.h/.cpp) bit for bit: same MQ register scaling and byte handling,
 * same contexts (T.800 Tables D.1-D.4), same MSB-plane rule and reconstruction bits; RESET,
 * TERMALL, SEGSYM and CAUSAL follow T.800 Annex D.
 *
 * The per-lane machine (struct Lane and its functions) compiles for the host too, so the
 * CPU tests can check it block by block against the oracle.
 */
#pragma once
#include <cstdint>

#include "plan.h"

#if defined(__CUDACC__)
#define J2K_LHD __host__ __device__ __forceinline__
#else
#define J2K_LHD inline
#endif

namespace j2k_lanes {

constexpr int LANES = 32;
constexpr int MAXW = 64, MAXH = 64, MAXS = MAXH / 4;

J2K_LHD int clz32(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __clz(x);
#else
  return x ? __builtin_clz(x) : 32;
#endif
}
J2K_LHD int ffs32(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __ffs(x);
#else
  return __builtin_ffs((int)x);
#endif
}
J2K_LHD int ffs64(uint64_t x) {
#ifdef __CUDA_ARCH__
  return __ffsll((long long)x);
#else
  return __builtin_ffsll((long long)x);
#endif
}
J2K_LHD uint32_t ldg32(const uint32_t *p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}
J2K_LHD void xor32(int32_t *p, uint32_t v) {
#ifdef __CUDA_ARCH__
  atomicXor(reinterpret_cast<unsigned int *>(p), v);
#else
  *reinterpret_cast<uint32_t *>(p) ^= v;
#endif
}

enum { C_SIG = 0, C_RUN = 9, C_SIGN = 10, C_MAG = 15, C_UNI = 18, N_CTX = 19 };
enum { P_SP = 0, P_MR = 1, P_CU = 2 };
// pending decision of a lane
enum { K_ZC = 0, K_SIGN, K_MR, K_RUN, K_UNI0, K_UNI1, K_SEGSYM, K_DONE };

// Shared tables, built on the host (build_lane_tables) and copied to shared memory per CTA.
struct LaneTables {
  uint32_t mq[94];       // context word of probability state s (= index * 2 + MPS)
  uint32_t next[94][2];  // word after a renormalising MPS [0] / LPS [1] decision in state s
  uint8_t zc[3][256];    // zero-coding context by 8-neighbour index (zc_index) for LL/LH, HL, HH
  uint8_t sc[256];       // (sign context << 1) | xor bit by sign_index
};

// per-lane view of the interleaved state
struct LaneMem {
  uint64_t *sig, *chi, *pi, *rho, *nb, *sc;
  uint32_t *cx;
  int lane;
  J2K_LHD uint64_t &SIG(int c) const { return sig[c * LANES + lane]; }
  J2K_LHD uint64_t &CHI(int c) const { return chi[c * LANES + lane]; }
  J2K_LHD uint64_t &PI(int c) const { return pi[c * LANES + lane]; }
  J2K_LHD uint64_t &RHO(int c) const { return rho[c * LANES + lane]; }
  J2K_LHD uint64_t &NB(int s) const { return nb[s * LANES + lane]; }
  J2K_LHD uint64_t &SC(int s) const { return sc[s * LANES + lane]; }
  J2K_LHD uint32_t &CX(int i) const { return cx[i * LANES + lane]; }
};

// bytes of the interleaved state of one warp (LANES blocks)
constexpr int STATE_U64 = 4 * MAXW + 2 * MAXS;  // sig, chi, pi, rho, nb, sc per lane
constexpr int WARP_BYTES = (STATE_U64 * 8 + N_CTX * 4) * LANES;

// Registers of one lane: MQ decoder, block, position in the pass, and the current stripe
// column's neighbourhood.  Windows: bit 0 = the row above the stripe, bits 1-4 = the
// stripe's rows, bit 5 = the row below (cleared in CAUSAL blocks), for the columns left of,
// at and right of the current one.
struct Lane {
  int32_t A, C, t, T;
  uint32_t ap, aend;  // byte position and segment end, counted from `w`
  const uint32_t *w;  // the segment's first byte rounded down to a 4-byte boundary
  uint32_t cur, nxt;  // the word holding byte ap and the one after it
  int32_t *base;      // the block's first sample in the coefficient buffer
  uint32_t stride;
  const uint8_t *data;
  const uint32_t *segl;
  uint32_t data_len, seg_pos;
  int seg_idx, nseg;
  int bw, stripes, flags, band;
  uint32_t lastrows;  // rows present in the last stripe
  uint64_t wmask;     // columns present
  int num_passes, kp, type, p;
  int s, c, wc, k, kind, ctx, flip, run, status;  // wc: the column the windows hold
  uint32_t e;  // context word of the pending decision, loaded when the decision is set up
  uint32_t rows, vrows;
  uint32_t eL, eC, eR, xL, xC, xR;
  uint32_t pin, rin, dirty;  // pi / rho nibbles of the current column, bits set during the visit
  uint64_t nbs, scs;         // nb / sc of the current stripe
};

// ---- MQ decoder (bmi_mq_decoder.h:52-169, bmi_mq_decoder.cpp:186-219), one per lane
J2K_LHD int mq_byte(const Lane &m) { return m.ap < m.aend ? (int)((m.cur >> ((m.ap & 3) * 8)) & 0xFF) : 0xFF; }
J2K_LHD void mq_advance(Lane &m) {
  m.ap++;
  if (!(m.ap & 3)) {
    m.cur = m.nxt;
    m.nxt = ldg32(m.w + (m.ap >> 2) + 1);
  }
}
// after a 0xFF byte the next byte carries 7 bits, unless it is a marker (> 0x8F), which is
// not consumed and reads as 0xFF with 8 bits
J2K_LHD void mq_fill(Lane &m) {
  const int b = mq_byte(m);
  const bool ff = m.T == 0xFF;
  const bool marker = ff && b > 0x8F;
  m.T = marker ? 0xFF : (ff ? b << 1 : b);
  if (!marker) mq_advance(m);
  m.t = (ff && !marker) ? 7 : 8;
  m.C += m.T;
}
// word loads reach up to 9 bytes past the segment; the code byte buffer carries 16 bytes of
// slack after its last segment
J2K_LHD void mq_init(Lane &m, const uint8_t *base, uint32_t len) {
  const uint32_t off = (uint32_t)((uintptr_t)base & 3);
  m.w = reinterpret_cast<const uint32_t *>(base - off);
  m.ap = off;
  m.aend = off + len;
  m.cur = ldg32(m.w);
  m.nxt = ldg32(m.w + 1);
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
J2K_LHD void mq_renorm(Lane &m) {
  int n = clz32((uint32_t)m.A) - 8;
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
// one decision on context slot L.ctx, whose word L.e holds (MQ_DECODE,
// bmi_mq_decoder.h:86-128)
J2K_LHD int decide(Lane &L, const LaneMem &M, const LaneTables &T) {
  const uint32_t e = L.e;
  const int32_t q = (int32_t)(e & 0x7FFFFFu);
  const int mps = (int)((e >> 23) & 1);
  L.A -= q;
  const bool ex = L.C < q;
  if (!ex && L.A >= 0x800000) {
    L.C -= q;
    return mps;
  }
  const bool lps = (L.A < q) != ex;
  if (ex) L.A = q;
  else L.C -= q;
  M.CX(L.ctx) = T.next[e >> 24][lps ? 1 : 0];
  mq_renorm(L);
  return mps ^ (int)lps;
}
J2K_LHD void init_contexts(const LaneMem &M, const LaneTables &T) {
  // bmi_mq_decoder.cpp:65-79: (state 0, MPS 0) except zero-coding context 0 -> state 4,
  // run length -> state 3; the run-position / segmentation symbols use a context pinned at
  // state 46 (the reference's fixed-Qe MQ_DECODE_START)
  for (int i = 0; i < N_CTX; ++i) M.CX(i) = T.mq[0];
  M.CX(C_SIG) = T.mq[4 << 1];
  M.CX(C_RUN) = T.mq[3 << 1];
  M.CX(C_UNI) = T.mq[46 << 1];
}

// ---- neighbourhoods
J2K_LHD uint32_t ext6(uint64_t col, int s, bool causal) {
  const uint32_t e = s == 0 ? (uint32_t)(col << 1) : (uint32_t)(col >> (4 * s - 1));
  return e & (causal ? 0x1Fu : 0x3Fu);
}
// 8-neighbour index of row k: bits 0-2 the left column's rows k-1..k+1, 3-5 the right
// column's, 6 the row above, 7 the row below
J2K_LHD int zc_index(uint32_t eL, uint32_t eC, uint32_t eR, int k) {
  return (int)(((eL >> k) & 7) | (((eR >> k) & 7) << 3) | (((eC >> k) & 1) << 6) | (((eC >> (k + 2)) & 1) << 7));
}
// sign index of row k: bit 0 sigma up, 1 chi up, 2 sigma down, 3 chi down, 4 sigma left,
// 5 chi left, 6 sigma right, 7 chi right
J2K_LHD int sign_index(const Lane &L, int k) {
  return (int)(((L.eC >> k) & 1) | (((L.xC >> k) & 1) << 1) | (((L.eC >> (k + 2)) & 1) << 2) |
               (((L.xC >> (k + 2)) & 1) << 3) | (((L.eL >> (k + 1)) & 1) << 4) | (((L.xL >> (k + 1)) & 1) << 5) |
               (((L.eR >> (k + 1)) & 1) << 6) | (((L.xR >> (k + 1)) & 1) << 7));
}
// rows of the current column each pass codes
J2K_LHD uint32_t sp_rows(const Lane &L) {
  const uint32_t m = L.eL | L.eC | L.eR;
  return (m | (m >> 1) | (m >> 2)) & ~(L.eC >> 1) & ~L.pin & L.vrows;
}
J2K_LHD uint32_t mr_rows(const Lane &L) { return (L.eC >> 1) & ~L.pin & L.vrows; }
J2K_LHD uint32_t cu_rows(const Lane &L) { return ~(L.eC >> 1) & ~L.pin & L.vrows; }

// context of the pending decision at row L.k
J2K_LHD void set_ctx(Lane &L, const LaneTables &T) {
  const int k = L.k;
  if (L.kind == K_MR) {
    const uint32_t nb = (((L.eL | L.eR) >> k) & 7) | ((L.eC >> k) & 5);
    L.ctx = C_MAG + (((L.rin >> k) & 1) ? 2 : (nb ? 1 : 0));
  } else if (L.kind == K_ZC) {
    L.ctx = C_SIG + T.zc[L.band][zc_index(L.eL, L.eC, L.eR, k)];
  } else {
    const int v = T.sc[sign_index(L, k)];
    L.ctx = C_SIGN + (v >> 1);
    L.flip = v & 1;
  }
}

// ---- pass walk
J2K_LHD void enter_stripe(Lane &L, const LaneMem &M, int s) {
  L.s = s;
  L.c = -1;
  L.wc = -2;
  L.nbs = M.NB(s);
  L.scs = M.SC(s);
  L.vrows = s == L.stripes - 1 ? L.lastrows : 0xFu;
}
// the windows of column c2 (shifted from the ones held when c2 is the next column)
J2K_LHD void load_windows(Lane &L, const LaneMem &M, int c2) {
  const bool causal = (L.flags & J2K_CB_CAUSAL) != 0;
  if (c2 == L.wc + 1) {
    L.eL = L.eC;
    L.xL = L.xC;
    L.eC = L.eR;
    L.xC = L.xR;
  } else {
    L.eL = c2 > 0 ? ext6(M.SIG(c2 - 1), L.s, causal) : 0u;
    L.xL = c2 > 0 ? ext6(M.CHI(c2 - 1), L.s, causal) : 0u;
    L.eC = ext6(M.SIG(c2), L.s, causal);
    L.xC = ext6(M.CHI(c2), L.s, causal);
  }
  L.eR = c2 + 1 < L.bw ? ext6(M.SIG(c2 + 1), L.s, causal) : 0u;
  L.xR = c2 + 1 < L.bw ? ext6(M.CHI(c2 + 1), L.s, causal) : 0u;
  L.wc = c2;
}
J2K_LHD void enter_column(Lane &L, const LaneMem &M, int c2) {
  load_windows(L, M, c2);
  L.c = c2;
  const int sh = 4 * L.s;
  L.pin = (uint32_t)(M.PI(c2) >> sh) & 0xFu;
  L.rin = L.type == P_MR ? (uint32_t)(M.RHO(c2) >> sh) & 0xFu : 0u;
  L.dirty = 0;
}
// leaving the current column: the significance pass records the rows it coded (pi), the
// refinement pass the rows it refined (rho); the cleanup pass, the last of the bit-plane,
// clears pi (bmi_block_decoder.cpp:571-573)
J2K_LHD void leave_column(Lane &L, const LaneMem &M) {
  const int sh = 4 * L.s;
  if (L.type == P_SP) {
    if (L.dirty) M.PI(L.c) |= (uint64_t)L.dirty << sh;
  } else if (L.type == P_MR) {
    if (L.dirty) M.RHO(L.c) |= (uint64_t)L.dirty << sh;
  } else if (L.pin) {
    M.PI(L.c) &= ~((uint64_t)0xF << sh);
  }
}

J2K_LHD bool seg_starts(int flags, int j) {
  return j == 0 || (flags & J2K_CB_TERMALL) != 0;  // BYPASS blocks are not decoded here
}
// start pass L.kp (T.800 D.3 order: cleanup first, then significance, refinement, cleanup
// per bit-plane); false when the block is finished or in error
J2K_LHD bool start_pass(Lane &L, const LaneMem &M) {
  if (L.kp >= L.num_passes) {
    L.kind = K_DONE;
    return false;
  }
  if (L.kp > 0 && ++L.type == 3) {
    L.type = 0;
    L.p--;
  }
  if (L.p < 0) {
    L.status = 2;
    L.kind = K_DONE;
    return false;
  }
  if (seg_starts(L.flags, L.kp)) {
    uint32_t len;
    if (L.flags & J2K_CB_TERMALL) {
      if (L.seg_idx >= L.nseg) {
        L.status = 3;
        L.kind = K_DONE;
        return false;
      }
      len = ldg32(L.segl + L.seg_idx);
      L.seg_idx++;
    } else {
      len = L.data_len;
    }
    if (L.seg_pos + len > L.data_len) {
      L.status = 4;
      L.kind = K_DONE;
      return false;
    }
    mq_init(L, L.data + L.seg_pos, len);
    L.seg_pos += len;
  }
  L.kp++;
  enter_stripe(L, M, 0);
  return true;
}
// after a pass and its segmentation symbols: context reset, then the next pass
J2K_LHD bool finish_pass(Lane &L, const LaneMem &M, const LaneTables &T) {
  if (L.flags & J2K_CB_RESET) init_contexts(M, T);
  return start_pass(L, M);
}

// Move to the next pending decision after the current column: the next column of the
// stripe with work for this pass, then the next stripe, then the next pass.
J2K_LHD void advance(Lane &L, const LaneMem &M, const LaneTables &T) {
  if (L.c >= 0) leave_column(L, M);
  for (;;) {
    int c2;
    if (L.type == P_CU) {
      c2 = L.c + 1 < L.bw ? L.c + 1 : -1;
      if (c2 >= 0 && L.vrows == 0xFu && !((L.nbs >> c2) & 1)) {
        // run-mode columns from c2 on whose run-length symbols would all decode as MPS
        // (insignificant) without renormalisation (C >= n*Qe and A - n*Qe >= 0x8000,
        // scaled) are consumed in one step: A -= n*Qe, C -= n*Qe
        const uint32_t e = M.CX(C_RUN);
        const int32_t q = (int32_t)(e & 0x7FFFFFu);
        const int32_t m = L.A - 0x800000 < L.C ? L.A - 0x800000 : L.C;
        if (!((e >> 23) & 1) && m >= q) {
          const uint64_t z = (~L.nbs & L.wmask) >> c2;  // run-mode columns from c2 on (bit 0 set)
          int n = ~z ? ffs64(~z) - 1 : 64 - c2;
          if ((int64_t)n * q > m) n = m / q;
          L.A -= n * q;
          L.C -= n * q;
          L.c = c2 + n - 1;
          continue;
        }
      }
    } else {
      const uint64_t above = L.c >= 63 ? 0ull : (~0ull << (L.c + 1));
      const uint64_t cand = (L.type == P_SP ? L.nbs : L.scs) & L.wmask & above;
      c2 = cand ? ffs64(cand) - 1 : -1;
    }
    if (c2 < 0) {
      if (L.s + 1 < L.stripes) {
        enter_stripe(L, M, L.s + 1);
        continue;
      }
      // end of the pass
      if (L.type == P_CU && (L.flags & J2K_CB_SEGSYM)) {
        L.kind = K_SEGSYM;
        L.ctx = C_UNI;
        L.run = 4;
        return;
      }
      if (!finish_pass(L, M, T)) return;
      continue;
    }
    if (L.type == P_CU && L.vrows == 0xFu && !((L.nbs >> c2) & 1)) {
      // run mode: the four rows insignificant, with insignificant neighbours, so not coded
      // by the significance pass either (pi clear); the windows are loaded only if the run
      // is interrupted by a significant sample
      L.c = c2;
      L.pin = L.rin = L.dirty = 0;
      L.kind = K_RUN;
      L.ctx = C_RUN;
      L.rows = 0xFu;
      return;
    }
    enter_column(L, M, c2);
    uint32_t rows;
    if (L.type == P_SP) rows = sp_rows(L);
    else if (L.type == P_MR) rows = mr_rows(L);
    else rows = cu_rows(L);
    if (rows) {
      L.rows = rows;
      L.k = ffs32(rows) - 1;
      L.kind = L.type == P_MR ? K_MR : K_ZC;
      set_ctx(L, T);
      return;
    }
    leave_column(L, M);
  }
}

// the next row of the current column (a significance-pass row may have become eligible
// through a new significant neighbour above it), else advance
J2K_LHD void next_row(Lane &L, const LaneMem &M, const LaneTables &T) {
  const uint32_t rows = (L.type == P_SP ? sp_rows(L) : L.rows) & (0xEu << L.k);
  if (rows) {
    L.rows = rows;
    L.k = ffs32(rows) - 1;
    L.kind = L.type == P_MR ? K_MR : K_ZC;
    set_ctx(L, T);
    return;
  }
  advance(L, M, T);
}

// row L.k of the current column becomes significant with sign `sym`
J2K_LHD void become_significant(Lane &L, const LaneMem &M, int sym) {
  const int k = L.k, r = 4 * L.s + k;
  const uint64_t bit = 1ull << r;
  M.SIG(L.c) |= bit;
  if (sym) M.CHI(L.c) |= bit;
  L.eC |= 2u << k;
  L.xC |= (uint32_t)sym << (k + 1);
  const uint64_t cm = L.c == 0 ? 3ull : (7ull << (L.c - 1));
  L.nbs |= cm;
  M.NB(L.s) = L.nbs;
  // the neighbouring stripes see row 0 (from above, except in CAUSAL blocks) and row 3
  if (k == 0 && L.s > 0 && !(L.flags & J2K_CB_CAUSAL)) M.NB(L.s - 1) |= cm;
  if (k == 3 && L.s + 1 < L.stripes) M.NB(L.s + 1) |= cm;
  M.SC(L.s) |= 1ull << L.c;
  L.base[(size_t)r * L.stride + L.c] = (int32_t)(((uint32_t)sym << 31) + (1u << L.p) + ((1u << L.p) >> 1));
}

// The outcome `d` of the pending decision; then the next pending decision.
J2K_LHD void lane_apply(Lane &L, const LaneMem &M, const LaneTables &T, int d) {
  switch (L.kind) {
    case K_ZC:
      if (L.type == P_SP) {
        L.pin |= 1u << L.k;
        L.dirty |= 1u << L.k;
      }
      if (d) {
        L.kind = K_SIGN;
        set_ctx(L, T);
        return;
      }
      break;
    case K_SIGN:
      become_significant(L, M, d ^ L.flip);
      break;
    case K_MR: {
      const int r = 4 * L.s + L.k;
      xor32(L.base + (size_t)r * L.stride + L.c, ((1u - (uint32_t)d) << L.p) | ((1u << L.p) >> 1));
      L.rin |= 1u << L.k;
      L.dirty |= 1u << L.k;
      break;
    }
    case K_RUN:
      if (!d) {  // the whole column stays insignificant
        advance(L, M, T);
        return;
      }
      L.kind = K_UNI0;
      L.ctx = C_UNI;
      return;
    case K_UNI0:
      L.run = d;
      L.kind = K_UNI1;
      return;
    case K_UNI1:
      // the first significant row of the run column: its sign follows directly, then the
      // rows below it are coded one by one
      L.k = L.run * 2 + d;
      L.kind = K_SIGN;
      if (L.wc != L.c) load_windows(L, M, L.c);
      set_ctx(L, T);
      return;
    default:  // K_SEGSYM
      if (--L.run > 0) return;
      if (finish_pass(L, M, T)) advance(L, M, T);
      return;
  }
  next_row(L, M, T);
}

// One MQ decision of a lane with a pending decision, then the next pending decision and
// its context word (read now, so the load overlaps the rest of the warp's loop trip).
J2K_LHD void lane_step(Lane &L, const LaneMem &M, const LaneTables &T) {
  lane_apply(L, M, T, decide(L, M, T));
  L.e = M.CX(L.ctx);
}

// MSB plane and pass count (bmi_block_decoder.cpp:603-622, :708-711)
J2K_LHD void block_planes(const j2k_cblk &cb, int &bit_plane, int &num_passes) {
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

// Start decoding block `cb` into `base` (stride cb.out_stride) on a lane whose state
// bitmaps are clear; the lane's first decision is pending afterwards (or it is done).
J2K_LHD void lane_begin(Lane &L, const LaneMem &M, const LaneTables &T, const j2k_cblk &cb, const uint8_t *bytes,
                        const uint32_t *seglens, int32_t *base) {
  L.base = base;
  L.stride = cb.out_stride;
  L.data = bytes + cb.data_off;
  L.segl = seglens + cb.seg_off;
  L.data_len = cb.data_len;
  L.seg_pos = 0;
  L.seg_idx = 0;
  L.nseg = cb.nseg;
  L.bw = cb.w;
  L.stripes = (cb.h + 3) >> 2;
  L.lastrows = (cb.h & 3) ? (1u << (cb.h & 3)) - 1u : 0xFu;
  L.wmask = cb.w >= 64 ? ~0ull : ((1ull << cb.w) - 1ull);
  L.flags = cb.flags;
  L.band = cb.band == 3 ? 2 : (cb.band == 1 ? 1 : 0);
  L.status = 0;
  L.A = L.C = L.t = L.T = 0;
  L.ap = L.aend = L.cur = L.nxt = 0;
  L.w = seglens;  // any readable address until the first segment starts
  L.c = -1;
  L.wc = -2;
  L.k = 0;
  L.ctx = 0;
  L.pin = L.rin = L.dirty = 0;
  L.eL = L.eC = L.eR = L.xL = L.xC = L.xR = 0;
  block_planes(cb, L.p, L.num_passes);
  init_contexts(M, T);
  L.type = P_CU;
  L.kp = 0;
  if (L.num_passes > 0 && 30 - (int)cb.missing <= 0) {
    L.status = 1;
    L.kind = K_DONE;
    return;
  }
  if (start_pass(L, M)) advance(L, M, T);
  L.e = M.CX(L.ctx);
}

// Whether block `cb` is decoded by the lane form: 64x64 at most, no raw (bypass) segments.
J2K_LHD bool lane_eligible(const j2k_cblk &cb) {
  return cb.w >= 1 && cb.h >= 1 && cb.w <= MAXW && cb.h <= MAXH && !(cb.flags & J2K_CB_BYPASS);
}

// ---- host: tables
inline void build_lane_tables(LaneTables &T) {
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
  auto word = [](int s) { return ((uint32_t)QE[s >> 1] << 8) | ((uint32_t)(s & 1) << 23) | ((uint32_t)s << 24); };
  for (int s = 0; s < 94; ++s) {
    const int idx = s >> 1, mps = s & 1;
    const int sw = QE[idx] == 0x5601 && NLPS[idx] != 46;  // T.800 Table C.2 SWITCH (states 0, 6, 14)
    T.mq[s] = word(s);
    T.next[s][0] = word(NMPS[idx] << 1 | mps);
    T.next[s][1] = word(NLPS[idx] << 1 | (mps ^ sw));
  }
  // T.800 Table D.1 from the horizontal / vertical / diagonal counts of a zc_index
  for (int band = 0; band < 3; ++band)
    for (int nb = 0; nb < 256; ++nb) {
      int h = ((nb >> 1) & 1) + ((nb >> 4) & 1);
      int v = ((nb >> 6) & 1) + ((nb >> 7) & 1);
      const int d = (nb & 1) + ((nb >> 2) & 1) + ((nb >> 3) & 1) + ((nb >> 5) & 1);
      int c;
      if (band == 2) {  // HH
        const int hv = h + v;
        if (d >= 3) c = 8;
        else if (d == 2) c = hv >= 1 ? 7 : 6;
        else if (d == 1) c = hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
        else c = hv >= 2 ? 2 : hv;
      } else {
        if (band == 1) {  // HL: horizontal and vertical roles exchanged
          const int x = h;
          h = v;
          v = x;
        }
        if (h == 2) c = 8;
        else if (h == 1) c = v >= 1 ? 7 : (d >= 1 ? 6 : 5);
        else if (v == 2) c = 4;
        else if (v == 1) c = 3;
        else c = d >= 2 ? 2 : d;
      }
      T.zc[band][nb] = (uint8_t)c;
    }
  // T.800 Tables D.2 / D.3
  for (int i = 0; i < 256; ++i) {
    auto contrib = [&](int sb, int xb) { return ((i >> sb) & 1) ? (((i >> xb) & 1) ? -1 : 1) : 0; };
    int H = contrib(4, 5) + contrib(6, 7);
    int V = contrib(0, 1) + contrib(2, 3);
    H = H < -1 ? -1 : (H > 1 ? 1 : H);
    V = V < -1 ? -1 : (V > 1 ? 1 : V);
    int x = 0;
    if (H < 0 || (H == 0 && V < 0)) {
      H = -H;
      V = -V;
      x = 1;
    }
    const int c = (H == 1) ? (V == 1 ? 4 : (V == 0 ? 3 : 2)) : (V == 1 ? 1 : 0);
    T.sc[i] = (uint8_t)(c << 1 | x);
  }
}

#if defined(__CUDACC__)
constexpr int CTA_WARPS = 3;
constexpr size_t TABLE_BYTES = (sizeof(LaneTables) + 15) & ~(size_t)15;
constexpr size_t CTA_SMEM = TABLE_BYTES + (size_t)CTA_WARPS * WARP_BYTES;

__device__ __forceinline__ int32_t signmag_to_int(int32_t v) {
  // FETCHPIXEL_INT, bmi_cpu_dwt_decoder.cpp:2287
  return (v & 0x80000000) ? ((v - 1) ^ 0x7FFFFFFF) : (v & 0x7FFFFFFF);
}
__device__ __forceinline__ int32_t place53(int32_t v, int numbps) {
  // dec_t1_comp.cpp:341-366
  int sh = 31 - numbps;
  sh = sh < 0 ? 0 : (sh > 31 ? 31 : sh);
  return v < 0 ? -(int32_t)((uint32_t)(v & 0x7FFFFFFF) >> sh) : (int32_t)((uint32_t)v >> sh);
}

// Persistent kernel: CTA_WARPS warps per CTA, one CTA per SM; every lane pulls code-blocks
// from the queue (`order`, longest first) and decodes them one decision per loop trip.  When
// a lane finishes, the warp rewrites that block in place (raw sign-magnitude -> dequantised
// float for 9/7, shifted integer for 5/3; coalesced rows; samples whose significance bit
// is clear were never written and become 0), clears its state and gives it the next block.
__global__ void __launch_bounds__(CTA_WARPS * 32, 1)
    t1_kernel_lanes(const j2k_cblk *__restrict__ cbs, const uint32_t *__restrict__ order, int n,
                    int *__restrict__ counter, const uint8_t *__restrict__ bytes, const uint32_t *__restrict__ seglens,
                    void *__restrict__ coef, uint16_t *__restrict__ status, const LaneTables *__restrict__ gtab) {
  extern __shared__ __align__(16) uint8_t smem[];
  LaneTables &T = *reinterpret_cast<LaneTables *>(smem);
  for (int i = threadIdx.x; i < (int)(sizeof(LaneTables) / 4); i += blockDim.x)
    reinterpret_cast<uint32_t *>(smem)[i] = reinterpret_cast<const uint32_t *>(gtab)[i];
  __syncthreads();
  const unsigned FULL = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  LaneMem M;
  M.sig = reinterpret_cast<uint64_t *>(smem + TABLE_BYTES + (size_t)warp * WARP_BYTES);
  M.chi = M.sig + MAXW * LANES;
  M.pi = M.chi + MAXW * LANES;
  M.rho = M.pi + MAXW * LANES;
  M.nb = M.rho + MAXW * LANES;
  M.sc = M.nb + MAXS * LANES;
  M.cx = reinterpret_cast<uint32_t *>(M.sc + MAXS * LANES);
  M.lane = lane;
  Lane L;
  L.kind = K_DONE;
  L.status = 0;
  bool have = false, live = true, first = true;  // holding a block; the queue may have more
  uint32_t ci = 0;
  for (;;) {
    // finished blocks: rewrite, status
    uint32_t fin = __ballot_sync(FULL, have && L.kind == K_DONE);
    if (fin) {
      __threadfence();
      __syncwarp();
    }
    while (fin) {
      const int j = __ffs(fin) - 1;
      fin &= fin - 1;
      const uint32_t cj = __shfl_sync(FULL, ci, j);
      const j2k_cblk cb = cbs[cj];
      int32_t *blk = reinterpret_cast<int32_t *>(coef) + cb.out_off;
      const int w = cb.w, h = cb.h;
      const bool irrev = (cb.flags & J2K_CB_IRREV) != 0;
      const uint64_t s0 = lane < w ? M.sig[lane * LANES + j] : 0ull;
      const uint64_t s1 = lane + 32 < w ? M.sig[(lane + 32) * LANES + j] : 0ull;
      for (int y = 0; y < h; ++y) {
        int32_t *r = blk + (size_t)y * cb.out_stride;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          const int x = lane + 32 * half;
          if (x >= w) continue;
          const int32_t v = (((half ? s1 : s0) >> y) & 1) ? __ldcg(r + x) : 0;
          if (irrev) *reinterpret_cast<float *>(r + x) = __fmul_rn((float)signmag_to_int(v), cb.gain);
          else r[x] = place53(v, cb.mb);
        }
      }
      if (lane == j) {
        status[cj] = (uint16_t)L.status;
        have = false;
      }
    }
    // next blocks: first one block per lane, dealt round the warps of the grid (so a short
    // queue still spreads over every SM), then from the shared counter
    bool got = false;
    if (!have && live) {
      const int lanes_total = gridDim.x * CTA_WARPS * 32;
      const int idx = first ? lane * (gridDim.x * CTA_WARPS) + blockIdx.x * CTA_WARPS + warp
                            : lanes_total + atomicAdd(counter, 1);
      first = false;
      if (idx < n) {
        ci = order[idx];
        got = true;
      } else {
        live = false;
      }
    }
    const uint32_t fresh = __ballot_sync(FULL, got);
    if (!__ballot_sync(FULL, have || got)) break;
    for (uint32_t m = fresh; m; m &= m - 1) {
      const int j = __ffs(m) - 1;
      for (int e = lane; e < STATE_U64; e += 32) M.sig[e * LANES + j] = 0ull;
    }
    __syncwarp();
    if (got) {
      const j2k_cblk cb = cbs[ci];
      lane_begin(L, M, T, cb, bytes, seglens, reinterpret_cast<int32_t *>(coef) + cb.out_off);
      have = true;
    }
    // decode until a lane finishes its block
    while (!__ballot_sync(FULL, have && L.kind == K_DONE)) {
      if (have) lane_step(L, M, T);
    }
  }
}
#endif

}  // namespace j2k_lanes
