/*
 * j2k_encoder.cpp — minimal JPEG 2000 Part-1 codestream writer (ITU-T T.800).
 *
 * Test and benchmark input generator: the reference carries no encoder
 * (decoder/core/src/encoderconcrete.cpp is an interface shell) and no sample codestreams,
 * so every stream decoded by this project is written here from a seeded image.
 *
 * Pipeline per tile: DC level shift -> forward RCT/ICT -> forward 5/3 (integer) or 9/7
 * (double) lifting DWT (vertical then horizontal, the inverse order of the decoder's
 * HDWT-then-VDWT, decoder/codec/src/bmi_cpu_dwt_decoder.cpp:1375-1772) -> deadzone
 * quantisation -> EBCOT Tier-1 with the MQ coder -> slope-threshold layer formation ->
 * Tier-2 packets with tag trees -> markers.
 */
#include "j2k_encoder.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// ----------------------------------------------------------------------------------------
// MQ coder probability estimation table, T.800 Table C.2 (Qe, NMPS, NLPS, SWITCH).
// The same 47 states appear in the reference decoder (bmi_mq_decoder.h:194-203,
// bmi_mq_decoder.cpp:37-42): the table is part of the standard, so it is restated here.
// ----------------------------------------------------------------------------------------
struct QeRow {
  uint16_t qe;
  uint8_t nmps, nlps, sw;
};
const QeRow kQe[47] = {
    {0x5601, 1, 1, 1},   {0x3401, 2, 6, 0},   {0x1801, 3, 9, 0},   {0x0AC1, 4, 12, 0},
    {0x0521, 5, 29, 0},  {0x0221, 38, 33, 0}, {0x5601, 7, 6, 1},   {0x5401, 8, 14, 0},
    {0x4801, 9, 14, 0},  {0x3801, 10, 14, 0}, {0x3001, 11, 17, 0}, {0x2401, 12, 18, 0},
    {0x1C01, 13, 20, 0}, {0x1601, 29, 21, 0}, {0x5601, 15, 14, 1}, {0x5401, 16, 14, 0},
    {0x5101, 17, 15, 0}, {0x4801, 18, 16, 0}, {0x3801, 19, 17, 0}, {0x3401, 20, 18, 0},
    {0x3001, 21, 19, 0}, {0x2801, 22, 19, 0}, {0x2401, 23, 20, 0}, {0x2201, 24, 21, 0},
    {0x1C01, 25, 22, 0}, {0x1801, 26, 23, 0}, {0x1601, 27, 24, 0}, {0x1401, 28, 25, 0},
    {0x1201, 29, 26, 0}, {0x1101, 30, 27, 0}, {0x0AC1, 31, 28, 0}, {0x09C1, 32, 29, 0},
    {0x08A1, 33, 30, 0}, {0x0521, 34, 31, 0}, {0x0441, 35, 32, 0}, {0x02A1, 36, 33, 0},
    {0x0221, 37, 34, 0}, {0x0141, 38, 35, 0}, {0x0111, 39, 36, 0}, {0x0085, 40, 37, 0},
    {0x0049, 41, 38, 0}, {0x0025, 42, 39, 0}, {0x0015, 43, 40, 0}, {0x0009, 44, 41, 0},
    {0x0005, 45, 42, 0}, {0x0001, 45, 43, 0}, {0x5601, 46, 46, 0}};

// context numbering used by this writer: 0-8 zero coding, 9-13 sign, 14-16 refinement,
// 17 run-length, 18 uniform
enum { CTX_ZC = 0, CTX_SC = 9, CTX_MR = 14, CTX_RL = 17, CTX_UNI = 18, NUM_CTX = 19 };

struct CtxState {
  uint8_t idx, mps;
};

void reset_contexts(CtxState *cx) {
  for (int i = 0; i < NUM_CTX; ++i) cx[i] = {0, 0};
  cx[CTX_ZC].idx = 4;
  cx[CTX_RL].idx = 3;
  cx[CTX_UNI].idx = 46;
}

// T.800 C.2 encoder (software conventions, registers A, C, CT; byte buffer with a leading
// dummy byte that plays the role of the byte before the segment).
struct MqEncoder {
  uint32_t A = 0x8000, C = 0;
  int CT = 12;
  std::vector<uint8_t> buf;  // buf[0] is the dummy byte
  void init() {
    A = 0x8000;
    C = 0;
    CT = 12;
    buf.assign(1, 0);
  }
  size_t emitted() const { return buf.size() - 1; }
  void byteout() {
    uint8_t &B = buf.back();
    if (B == 0xFF) {
      buf.push_back((uint8_t)(C >> 20));
      C &= 0xFFFFF;
      CT = 7;
    } else if (C < 0x8000000) {
      buf.push_back((uint8_t)(C >> 19));
      C &= 0x7FFFF;
      CT = 8;
    } else {
      B = (uint8_t)(B + 1);
      if (B == 0xFF) {
        C &= 0x7FFFFFF;
        buf.push_back((uint8_t)(C >> 20));
        C &= 0xFFFFF;
        CT = 7;
      } else {
        buf.push_back((uint8_t)(C >> 19));
        C &= 0x7FFFF;
        CT = 8;
      }
    }
  }
  void renorm() {
    do {
      A <<= 1;
      C <<= 1;
      if (--CT == 0) byteout();
    } while ((A & 0x8000) == 0);
  }
  void encode(CtxState &cx, int bit) {
    const QeRow &r = kQe[cx.idx];
    uint32_t qe = r.qe;
    A -= qe;
    if (bit == cx.mps) {
      if ((A & 0x8000) == 0) {
        if (A < qe)
          A = qe;
        else
          C += qe;
        cx.idx = r.nmps;
        renorm();
      } else {
        C += qe;
      }
    } else {
      if (A < qe)
        C += qe;
      else
        A = qe;
      if (r.sw) cx.mps ^= 1;
      cx.idx = r.nlps;
      renorm();
    }
  }
  // T.800 C.2.9 FLUSH; returns the segment bytes
  void flush(std::vector<uint8_t> &out) {
    uint32_t tempc = C + A;
    C |= 0xFFFF;
    if (C >= tempc) C -= 0x8000;
    C <<= CT;
    byteout();
    C <<= CT;
    byteout();
    size_t n = buf.size();
    if (buf[n - 1] == 0xFF) --n;
    out.insert(out.end(), buf.begin() + 1, buf.begin() + n);
  }
};

// raw (bypass) bit packer with 0xFF bit stuffing
struct RawEncoder {
  std::vector<uint8_t> buf;
  uint32_t c = 0;
  int ct = 8;
  void init() {
    buf.clear();
    c = 0;
    ct = 8;
  }
  void put(int bit) {
    --ct;
    c |= (uint32_t)(bit & 1) << ct;
    if (ct == 0) {
      buf.push_back((uint8_t)c);
      ct = (c == 0xFF) ? 7 : 8;
      c = 0;
    }
  }
  size_t bytes_for_bits() const {
    size_t n = buf.size();
    if (ct != 8 && !(ct == 7 && !buf.empty() && buf.back() == 0xFF && c == 0)) ++n;
    return n;
  }
  void flush(std::vector<uint8_t> &out) {
    bool partial = (ct != 8) && !(ct == 7 && !buf.empty() && buf.back() == 0xFF && c == 0);
    if (partial) buf.push_back((uint8_t)c);
    // a trailing 0xFF carries only 1-bits, which is what a decoder reads past the end
    while (!buf.empty() && buf.back() == 0xFF) buf.pop_back();
    out.insert(out.end(), buf.begin(), buf.end());
  }
};

// MQ decoder in the scaled-register form of the reference (A and C pre-shifted by 8, "S"
// counts synthesised 0xFF bytes; decoder/codec/src/bmi_mq_decoder.cpp:186-258).  Used
// here only to check that a truncated segment still decodes its passes.
struct MqVerifier {
  int32_t A, C, t, T;
  const uint8_t *p, *base;
  long maxidx;  // highest byte index read or peeked so far
  void touch() { maxidx = std::max(maxidx, (long)(p - base)); }
  void fill() {
    touch();
    if (T == 0xFF) {
      if (*p > 0x8F) {
        t = 8;
      } else {
        T = (int32_t)(*p++) << 1;
        t = 7;
      }
    } else {
      T = *p++;
      t = 8;
    }
    C += T;
  }
  void init(const uint8_t *buf) {
    p = base = buf;
    maxidx = -1;
    T = 0;
    C = 0;
    t = 0;
    fill();
    C <<= t;
    fill();
    C <<= 7;
    t -= 7;
    A = 0x800000;
  }
  void renorm_once() {
    if (!t) fill();
    A <<= 1;
    C <<= 1;
    --t;
  }
  int decode(CtxState &cx) {
    const QeRow &r = kQe[cx.idx];
    int32_t q = (int32_t)r.qe << 8;
    int ret = cx.mps;
    A -= q;
    if (C < q) {
      if (A < q) {
        cx.idx = r.nmps;
      } else {
        ret ^= 1;
        if (r.sw) cx.mps ^= 1;
        cx.idx = r.nlps;
      }
      A = q;
      do renorm_once();
      while (A < 0x800000);
    } else {
      C -= q;
      if (A < 0x800000) {
        if (A < q) {
          ret ^= 1;
          if (r.sw) cx.mps ^= 1;
          cx.idx = r.nlps;
        } else {
          cx.idx = r.nmps;
        }
        do renorm_once();
        while (A < 0x800000);
      }
    }
    return ret;
  }
};

// ----------------------------------------------------------------------------------------
// Tier-1 context formation (T.800 Annex D, Tables D.1, D.3, D.4)
// ----------------------------------------------------------------------------------------
struct ZcLut {
  uint8_t t[4][3][3][5];  // [band][h][v][d]
  ZcLut() {
    for (int b = 0; b < 4; ++b)
      for (int h = 0; h < 3; ++h)
        for (int v = 0; v < 3; ++v)
          for (int d = 0; d < 5; ++d) {
            int c;
            if (b == 3) {  // HH
              int hv = h + v;
              if (d >= 3) c = 8;
              else if (d == 2) c = hv >= 1 ? 7 : 6;
              else if (d == 1) c = hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
              else c = hv >= 2 ? 2 : (hv == 1 ? 1 : 0);
            } else {
              int H = h, V = v;
              if (b == 1) std::swap(H, V);  // HL: vertical neighbours are primary
              if (H == 2) c = 8;
              else if (H == 1) c = V >= 1 ? 7 : (d >= 1 ? 6 : 5);
              else if (V == 2) c = 4;
              else if (V == 1) c = 3;
              else c = d >= 2 ? 2 : (d == 1 ? 1 : 0);
            }
            t[b][h][v][d] = (uint8_t)c;
          }
  }
};
const ZcLut kZc;

// sign context: H, V in {-1,0,1} -> (context offset 0..4, xor bit)
inline void sign_ctx(int H, int V, int &ctx, int &xr) {
  if (H < 0) {
    H = -H;
    V = -V;
    xr = 1;
  } else if (H == 0 && V < 0) {
    V = -V;
    xr = 1;
  } else {
    xr = 0;
  }
  // now H in {0,1}; table D.3: (1,1)->13 (1,0)->12 (1,-1)->11 (0,1)->10 (0,0)->9
  if (H == 1) ctx = (V == 1) ? 4 : (V == 0 ? 3 : 2);
  else ctx = (V == 1) ? 1 : 0;
}

struct PassInfo {
  uint32_t end_len;  // bytes of the block stream needed to decode up to the end of this pass
  double dist;       // cumulative distortion reduction (weighted)
  int terminated;
};

struct CodeBlock {
  // geometry (band coordinates relative to the band origin of the tile-component)
  int x0, y0, w, h;
  int band;  // 0 LL, 1 HL, 2 LH, 3 HH
  int missing = 0;
  int nbits = 0;
  int npasses = 0;
  std::vector<uint8_t> data;
  std::vector<PassInfo> passes;
  // T2 state
  int incl_layer = 0;  // number of passes included after each layer is kept in layer_passes
  std::vector<int> layer_passes;
  int lblock = 3;
  bool included = false;
};

struct Band {
  int type;  // 0 LL 1 HL 2 LH 3 HH
  int x0, y0, x1, y1;  // band coordinates (absolute, T.800 B.5)
  int eps, mu;         // quantisation exponent / mantissa
  double delta;        // step in coefficient units (1 for reversible)
  double weight;       // synthesis energy gain * delta^2
  int Mb;
  int cbx0, cby0, ncbx, ncby;  // code-block grid
  std::vector<CodeBlock> cbs;
};

struct Resolution {
  int x0, y0, x1, y1;
  std::vector<Band> bands;
};

struct TileComp {
  int x0, y0, x1, y1;
  std::vector<Resolution> res;  // res[0] = LL_L ... res[L]
  std::vector<double> coef;     // transformed, row-major over the tile-component
};

struct Tile {
  int x0, y0, x1, y1;
  std::vector<TileComp> comps;
};

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline int ceil_div_pow2(int a, int l) { return (a + (1 << l) - 1) >> l; }
inline int floor_log2(uint32_t v) { return v ? 31 - __builtin_clz(v) : -1; }

// ---------------------------------------------------------------- forward wavelet ----
// 1-D forward 5/3 (T.800 F.4.8.1) on an even-origin signal with whole-sample symmetric
// extension.  x: n samples -> out: low ceil(n/2) then high floor(n/2).
void fwd53(const int64_t *x, int n, int64_t *low, int64_t *high) {
  if (n == 1) {
    low[0] = x[0];
    return;
  }
  int nl = (n + 1) / 2, nh = n / 2;
  auto X = [&](int i) -> int64_t {
    if (i >= n) i = 2 * (n - 1) - i;
    if (i < 0) i = -i;
    return x[i];
  };
  for (int i = 0; i < nh; ++i) {
    int64_t s = X(2 * i) + X(2 * i + 2);
    high[i] = x[2 * i + 1] - (s >= 0 ? s / 2 : -((-s + 1) / 2));
  }
  auto D = [&](int i) -> int64_t {
    if (i < 0) i = -1 - i;         // d[-1] = d[0]
    if (i >= nh) i = 2 * nh - 1 - i;  // mirror at the end (odd n)
    return high[i];
  };
  for (int i = 0; i < nl; ++i) {
    int64_t s = D(i - 1) + D(i) + 2;
    low[i] = x[2 * i] + (s >= 0 ? s / 4 : -((-s + 3) / 4));
  }
}

const double ALPHA = -1.586134342059924, BETA = -0.052980118572961, GAMMA = 0.882911075530934,
             DELTA = 0.443506852043971, KAPPA = 1.230174104914001;

// 1-D forward 9/7 (T.800 F.4.8.2), even origin, symmetric extension
void fwd97(const double *x, int n, double *low, double *high, std::vector<double> &tmp) {
  if (n == 1) {
    low[0] = x[0];
    return;
  }
  tmp.assign(x, x + n);
  double *y = tmp.data();
  auto at = [&](int i) -> double & {
    if (i < 0) i = -i;
    if (i >= n) i = 2 * (n - 1) - i;
    return y[i];
  };
  for (int i = 1; i < n; i += 2) y[i] += ALPHA * (at(i - 1) + at(i + 1));
  for (int i = 0; i < n; i += 2) y[i] += BETA * (at(i - 1) + at(i + 1));
  for (int i = 1; i < n; i += 2) y[i] += GAMMA * (at(i - 1) + at(i + 1));
  for (int i = 0; i < n; i += 2) y[i] += DELTA * (at(i - 1) + at(i + 1));
  for (int i = 0; i < n; ++i) {
    if (i & 1)
      high[i / 2] = y[i] * KAPPA;
    else
      low[i / 2] = y[i] / KAPPA;
  }
}

// inverse 1-D 9/7 (double) used only to measure synthesis energy gains of the bands
void inv97(const double *low, const double *high, int n, double *x) {
  if (n == 1) {
    x[0] = low[0];
    return;
  }
  std::vector<double> y(n);
  for (int i = 0; i < n; ++i) y[i] = (i & 1) ? high[i / 2] / KAPPA : low[i / 2] * KAPPA;
  auto at = [&](int i) -> double {
    if (i < 0) i = -i;
    if (i >= n) i = 2 * (n - 1) - i;
    return y[i];
  };
  for (int i = 0; i < n; i += 2) y[i] -= DELTA * (at(i - 1) + at(i + 1));
  for (int i = 1; i < n; i += 2) y[i] -= GAMMA * (at(i - 1) + at(i + 1));
  for (int i = 0; i < n; i += 2) y[i] -= BETA * (at(i - 1) + at(i + 1));
  for (int i = 1; i < n; i += 2) y[i] -= ALPHA * (at(i - 1) + at(i + 1));
  for (int i = 0; i < n; ++i) x[i] = y[i];
}

void inv53d(const double *low, const double *high, int n, double *x) {
  // real-valued 5/3 synthesis (no rounding) for energy gains
  if (n == 1) {
    x[0] = low[0];
    return;
  }
  int nl = (n + 1) / 2, nh = n / 2;
  (void)nl;
  std::vector<double> y(n);
  for (int i = 0; i < n; ++i) y[i] = (i & 1) ? high[i / 2] : low[i / 2];
  auto at = [&](int i) -> double {
    if (i < 0) i = -i;
    if (i >= n) i = 2 * (n - 1) - i;
    return y[i];
  };
  (void)nh;
  for (int i = 0; i < n; i += 2) y[i] -= (at(i - 1) + at(i + 1)) / 4.0;
  for (int i = 1; i < n; i += 2) y[i] += (at(i - 1) + at(i + 1)) / 2.0;
  for (int i = 0; i < n; ++i) x[i] = y[i];
}

// squared L2 norm of the 1-D synthesis basis of a band at `level` (1..L), low or high:
// an impulse in the middle of that band is synthesised back to full resolution
double synth_gain_1d(bool rev, int level, bool high) {
  const int N = 1 << std::max(level + 6, 10);
  int len_at[32];
  len_at[0] = N;
  for (int l = 1; l <= level; ++l) len_at[l] = (len_at[l - 1] + 1) / 2;
  std::vector<double> lo(len_at[level], 0.0), hi(len_at[level - 1] / 2, 0.0);
  if (high)
    hi[hi.size() / 2] = 1.0;
  else
    lo[lo.size() / 2] = 1.0;
  for (int l = level; l >= 1; --l) {
    int n = len_at[l - 1];
    std::vector<double> out(n);
    if (rev)
      inv53d(lo.data(), hi.data(), n, out.data());
    else
      inv97(lo.data(), hi.data(), n, out.data());
    lo.swap(out);
    if (l >= 2) hi.assign(len_at[l - 2] / 2, 0.0);
  }
  double e = 0;
  for (double v : lo) e += v * v;
  return e;
}

// ------------------------------------------------------------------- Tier-1 coder ----
struct T1Coder {
  int w, h, band, mode;
  std::vector<uint8_t> sig, vis, ref, sgn;  // (w+2)*(h+2) with a border
  std::vector<int32_t> mag;                 // |q|
  int stride;
  CtxState cx[NUM_CTX];
  MqEncoder mq;
  RawEncoder raw;
  std::vector<uint8_t> log_ctx, log_bit;  // MQ symbols of the current segment
  std::vector<size_t> pass_sym_end;       // symbol count at the end of each pass (segment-local)

  inline int at(int x, int y) const { return (y + 1) * stride + (x + 1); }

  void put(int c, int bit) {
    log_ctx.push_back((uint8_t)c);
    log_bit.push_back((uint8_t)bit);
    mq.encode(cx[c], bit);
  }

  // CAUSAL (T.800 D.7): the last row of a stripe sees the next stripe as insignificant
  bool below_cut(int y) const { return (mode & J2KENC_CAUSAL) && (y & 3) == 3; }
  void neighbours(int i, int y, int &hh, int &vv, int &dd) const {
    const int below = below_cut(y) ? 0 : 1;
    hh = sig[i - 1] + sig[i + 1];
    vv = sig[i - stride] + below * sig[i + stride];
    dd = sig[i - stride - 1] + sig[i - stride + 1] + below * (sig[i + stride - 1] + sig[i + stride + 1]);
  }
  void code_sign(int i, int y, bool rawmode) {
    int s = sgn[i];
    if (rawmode) {
      raw.put(s);
      return;
    }
    auto contrib = [&](int j) { return sig[j] ? (sgn[j] ? -1 : 1) : 0; };
    int H = contrib(i - 1) + contrib(i + 1);
    int V = contrib(i - stride) + (below_cut(y) ? 0 : contrib(i + stride));
    H = std::max(-1, std::min(1, H));
    V = std::max(-1, std::min(1, V));
    int c, xr;
    sign_ctx(H, V, c, xr);
    put(CTX_SC + c, s ^ xr);
  }

  void pass_sp(int p, bool rawmode, double &dist) {
    for (int y0 = 0; y0 < h; y0 += 4)
      for (int x = 0; x < w; ++x)
        for (int y = y0; y < std::min(y0 + 4, h); ++y) {
          int i = at(x, y);
          if (sig[i]) continue;
          int hh, vv, dd;
          neighbours(i, y, hh, vv, dd);
          if (hh + vv + dd == 0) continue;
          int bit = (mag[i] >> p) & 1;
          if (rawmode)
            raw.put(bit);
          else
            put(CTX_ZC + kZc.t[band][hh][vv][dd], bit);
          vis[i] = 1;
          if (bit) {
            code_sign(i, y, rawmode);
            sig[i] = 1;
            double m = mag[i], r = 1.5 * (double)(1 << p);
            dist += m * m - (m - r) * (m - r);
          }
        }
  }
  void pass_mr(int p, bool rawmode, double &dist) {
    for (int y0 = 0; y0 < h; y0 += 4)
      for (int x = 0; x < w; ++x)
        for (int y = y0; y < std::min(y0 + 4, h); ++y) {
          int i = at(x, y);
          if (!sig[i] || vis[i]) continue;
          int bit = (mag[i] >> p) & 1;
          if (rawmode) {
            raw.put(bit);
          } else {
            int c;
            if (ref[i]) {
              c = 2;
            } else {
              int hh, vv, dd;
              neighbours(i, y, hh, vv, dd);
              c = (hh + vv + dd) ? 1 : 0;
            }
            put(CTX_MR + c, bit);
          }
          ref[i] = 1;
          double m = mag[i];
          double before = (std::floor(m / (2 << p)) + 0.5) * (double)(2 << p);
          double after = (std::floor(m / (1 << p)) + 0.5) * (double)(1 << p);
          dist += (m - before) * (m - before) - (m - after) * (m - after);
        }
  }
  void code_cu_sample(int i, int y, int p, double &dist) {
    int hh, vv, dd;
    neighbours(i, y, hh, vv, dd);
    int bit = (mag[i] >> p) & 1;
    put(CTX_ZC + kZc.t[band][hh][vv][dd], bit);
    if (bit) {
      code_sign(i, y, false);
      sig[i] = 1;
      double m = mag[i], r = 1.5 * (double)(1 << p);
      dist += m * m - (m - r) * (m - r);
    }
  }
  void pass_cu(int p, double &dist) {
    for (int y0 = 0; y0 < h; y0 += 4)
      for (int x = 0; x < w; ++x) {
        int ye = std::min(y0 + 4, h);
        int ystart = y0;
        if (ye - y0 == 4) {
          bool run = true;
          for (int y = y0; y < ye && run; ++y) {
            int i = at(x, y);
            if (sig[i] || vis[i]) run = false;
            else {
              int hh, vv, dd;
              neighbours(i, y, hh, vv, dd);
              if (hh + vv + dd) run = false;
            }
          }
          if (run) {
            int r = -1;
            for (int y = y0; y < ye; ++y)
              if ((mag[at(x, y)] >> p) & 1) {
                r = y - y0;
                break;
              }
            if (r < 0) {
              put(CTX_RL, 0);
              continue;
            }
            put(CTX_RL, 1);
            put(CTX_UNI, (r >> 1) & 1);
            put(CTX_UNI, r & 1);
            int i = at(x, y0 + r);
            code_sign(i, y0 + r, false);
            sig[i] = 1;
            double m = mag[i], rr = 1.5 * (double)(1 << p);
            dist += m * m - (m - rr) * (m - rr);
            ystart = y0 + r + 1;
          }
        }
        for (int y = ystart; y < ye; ++y) {
          int i = at(x, y);
          if (sig[i] || vis[i]) continue;
          code_cu_sample(i, y, p, dist);
        }
      }
    if (mode & J2KENC_SEGSYM) {
      put(CTX_UNI, 1);
      put(CTX_UNI, 0);
      put(CTX_UNI, 1);
      put(CTX_UNI, 0);
    }
    std::fill(vis.begin(), vis.end(), 0);
  }

  // Replay the logged symbols of a finished MQ segment through a decoder and record, for
  // every pass end, the number of segment bytes the decoder has read or peeked at.  A
  // truncation at that length (decoder-side 0xFF 0xFF padding) decodes the same symbols.
  void safe_lengths(const uint8_t *seg, size_t len, std::vector<uint32_t> &out) {
    std::vector<uint8_t> b(seg, seg + len);
    b.push_back(0xFF);
    b.push_back(0xFF);
    b.push_back(0xFF);
    MqVerifier d;
    d.init(b.data());
    CtxState c[NUM_CTX];
    reset_contexts(c);
    out.assign(pass_sym_end.size(), 0);
    size_t k = 0;
    for (size_t pe = 0; pe < pass_sym_end.size(); ++pe) {
      for (; k < pass_sym_end[pe]; ++k) {
        int bit = d.decode(c[log_ctx[k]]);
        if (bit != log_bit[k]) std::abort();  // the coder and its replay disagree
      }
      out[pe] = (uint32_t)std::min<long>((long)len, d.maxidx + 1);
      if (mode & J2KENC_RESET) reset_contexts(c);
    }
  }

  void encode(const int32_t *q, int qstride, CodeBlock &cb, int Mb, double weight) {
    w = cb.w;
    h = cb.h;
    band = cb.band;
    stride = w + 2;
    size_t n = (size_t)(w + 2) * (h + 2);
    sig.assign(n, 0);
    vis.assign(n, 0);
    ref.assign(n, 0);
    sgn.assign(n, 0);
    mag.assign(n, 0);
    int32_t maxm = 0;
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        int32_t v = q[(size_t)y * qstride + x];
        int i = at(x, y);
        sgn[i] = v < 0;
        mag[i] = v < 0 ? -v : v;
        maxm = std::max(maxm, mag[i]);
      }
    cb.nbits = maxm ? floor_log2((uint32_t)maxm) + 1 : 0;
    cb.missing = Mb - cb.nbits;
    cb.data.clear();
    cb.passes.clear();
    if (!cb.nbits) {
      cb.npasses = 0;
      return;
    }
    const int npasses = 3 * cb.nbits - 2;
    cb.npasses = npasses;
    reset_contexts(cx);
    mq.init();
    log_ctx.clear();
    log_bit.clear();
    pass_sym_end.clear();
    size_t seg_start = 0;   // offset of the current segment in cb.data
    int seg_first_pass = 0;
    bool seg_raw = false;
    double dist = 0;
    std::vector<uint32_t> rel_len(npasses, 0);  // segment-relative truncation lengths
    for (int k = 0; k < npasses; ++k) {
      int type = (k == 0) ? 2 : (k - 1) % 3;  // 0 SP, 1 MR, 2 CU
      int p = cb.nbits - 1 - (k + 2) / 3;
      bool rawp = (mode & J2KENC_BYPASS) && k >= 10 && type != 2;
      bool new_seg = (k == 0) || (mode & J2KENC_TERMALL) ||
                     ((mode & J2KENC_BYPASS) && k >= 10 && type != 1);
      if (new_seg && k > 0) {
        // terminate the previous segment (already flushed at the end of pass k-1)
      }
      if (new_seg) {
        seg_start = cb.data.size();
        seg_first_pass = k;
        seg_raw = rawp;
        if (rawp)
          raw.init();
        else {
          mq.init();
          log_ctx.clear();
          log_bit.clear();
          pass_sym_end.clear();
        }
      }
      if (type == 0) pass_sp(p, rawp, dist);
      else if (type == 1) pass_mr(p, rawp, dist);
      else pass_cu(p, dist);
      if (!seg_raw) pass_sym_end.push_back(log_ctx.size());
      if (mode & J2KENC_RESET) reset_contexts(cx);
      // does the segment end after this pass?
      bool last = (k == npasses - 1);
      int ntype = (k + 1 - 1) % 3;
      bool next_new = !last && ((mode & J2KENC_TERMALL) ||
                                ((mode & J2KENC_BYPASS) && k + 1 >= 10 && ntype != 1));
      PassInfo pi;
      pi.dist = dist * weight;
      if (last || next_new) {
        if (seg_raw)
          raw.flush(cb.data);
        else
          mq.flush(cb.data);
        pi.terminated = 1;
        pi.end_len = (uint32_t)cb.data.size();
        // truncation lengths of the earlier passes of this segment
        size_t seg_len = cb.data.size() - seg_start;
        std::vector<uint32_t> safe;
        if (!seg_raw && k > seg_first_pass) safe_lengths(cb.data.data() + seg_start, seg_len, safe);
        uint32_t prevl = 0;
        for (int j = seg_first_pass; j < k; ++j) {
          uint32_t l = seg_raw ? rel_len[j] : safe[j - seg_first_pass];
          l = std::min<uint32_t>(std::max(l, prevl), (uint32_t)seg_len);
          // keep truncation points off a trailing 0xFF
          while (l > 0 && l < seg_len && cb.data[seg_start + l - 1] == 0xFF) ++l;
          prevl = l;
          cb.passes[j].end_len = (uint32_t)seg_start + l;
        }
      } else {
        pi.terminated = 0;
        rel_len[k] = seg_raw ? (uint32_t)raw.bytes_for_bits() : 0;
        pi.end_len = 0;
      }
      cb.passes.push_back(pi);
    }
  }
};

// ------------------------------------------------------------------- bit writer (T2) ---
struct BitWriter {
  std::vector<uint8_t> &out;
  uint32_t c = 0;
  int ct = 8;
  explicit BitWriter(std::vector<uint8_t> &o) : out(o) {}
  void put(int bit) {
    --ct;
    c |= (uint32_t)(bit & 1) << ct;
    if (ct == 0) {
      out.push_back((uint8_t)c);
      ct = (c == 0xFF) ? 7 : 8;
      c = 0;
    }
  }
  void put_bits(uint32_t v, int n) {
    for (int i = n - 1; i >= 0; --i) put((v >> i) & 1);
  }
  void flush() {
    if (ct != 8) {
      if (!(ct == 7 && c == 0 && !out.empty() && out.back() == 0xFF)) out.push_back((uint8_t)c);
      else out.push_back(0);  // byte after 0xFF
    }
    if (!out.empty() && out.back() == 0xFF) out.push_back(0);
    ct = 8;
    c = 0;
  }
};

struct TagTree {
  struct Node {
    int value, low, known, parent;
  };
  std::vector<Node> nodes;
  int nleaf = 0;
  void build(int w, int h) {
    nodes.clear();
    nleaf = w * h;
    std::vector<std::pair<int, int>> dims;
    int lw = w, lh = h;
    dims.push_back({lw, lh});
    while (lw > 1 || lh > 1) {
      lw = (lw + 1) / 2;
      lh = (lh + 1) / 2;
      dims.push_back({lw, lh});
    }
    int total = 0;
    std::vector<int> base;
    for (auto &d : dims) {
      base.push_back(total);
      total += d.first * d.second;
    }
    nodes.assign(total, {0, 0, 0, -1});
    for (size_t l = 0; l + 1 < dims.size(); ++l) {
      int dw = dims[l].first, dh = dims[l].second, pw = dims[l + 1].first;
      for (int y = 0; y < dh; ++y)
        for (int x = 0; x < dw; ++x) nodes[base[l] + y * dw + x].parent = base[l + 1] + (y / 2) * pw + x / 2;
    }
  }
  void set_values(const std::vector<int> &leaf) {
    for (auto &n : nodes) {
      n.value = 1 << 30;
      n.low = 0;
      n.known = 0;
    }
    for (int i = 0; i < nleaf; ++i) {
      int v = leaf[i];
      int j = i;
      while (j >= 0) {
        if (nodes[j].value > v) nodes[j].value = v;
        j = nodes[j].parent;
      }
    }
  }
  void encode(BitWriter &bw, int leaf, int threshold) {
    int stk[32], sp = 0;
    int node = leaf;
    while (nodes[node].parent >= 0) {
      stk[sp++] = node;
      node = nodes[node].parent;
    }
    int low = 0;
    for (;;) {
      Node &n = nodes[node];
      if (low > n.low) n.low = low;
      else low = n.low;
      while (low < threshold) {
        if (low >= n.value) {
          if (!n.known) {
            bw.put(1);
            n.known = 1;
          }
          break;
        }
        bw.put(0);
        ++low;
      }
      n.low = low;
      if (!sp) break;
      node = stk[--sp];
    }
  }
};

void put_u16(std::vector<uint8_t> &o, unsigned v) {
  o.push_back((uint8_t)(v >> 8));
  o.push_back((uint8_t)v);
}
void put_u32(std::vector<uint8_t> &o, uint32_t v) {
  put_u16(o, v >> 16);
  put_u16(o, v & 0xFFFF);
}

int seg_starts(int mode, int j) {
  int type = (j == 0) ? 2 : (j - 1) % 3;
  return j == 0 || (mode & J2KENC_TERMALL) || ((mode & J2KENC_BYPASS) && j >= 10 && type != 1);
}

}  // namespace

extern "C" void j2kenc_default_params(j2kenc_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->reversible = 1;
  p->levels = 5;
  p->cbw_exp = 6;
  p->cbh_exp = 6;
  p->num_layers = 1;
  p->progression = J2KENC_LRCP;
  p->use_mct = 1;
  p->base_step = 1.0 / 256.0;
}

extern "C" void j2kenc_free(void *p) { std::free(p); }

extern "C" int j2kenc_encode(const uint16_t *planes, int W, int H, int ncomp, int B,
                             const j2kenc_params *P, uint8_t **out, size_t *out_len) {
  if (!planes || !P || !out || !out_len) return -1;
  if (W <= 0 || H <= 0 || ncomp < 1 || ncomp > 4 || B < 1 || B > 16) return -2;
  const int L = P->levels;
  if (L < 0 || L > 10) return -3;
  if (P->cbw_exp < 2 || P->cbh_exp < 2 || P->cbw_exp + P->cbh_exp > 12) return -4;
  if (P->num_layers < 1 || P->num_layers > 32) return -5;
  const int TW = P->tile_w > 0 ? P->tile_w : W, TH = P->tile_h > 0 ? P->tile_h : H;
  if (P->tile_w > 0 && ((TW % (1 << L)) || (TH % (1 << L)))) return -7;  // even origins at all levels
  int dx[4], dy[4];
  for (int c = 0; c < 4; ++c) {
    dx[c] = P->sub_x[c] > 1 ? P->sub_x[c] : 1;
    dy[c] = P->sub_y[c] > 1 ? P->sub_y[c] : 1;
    if (dx[c] > 255 || dy[c] > 255) return -12;
    // tile-components start on even coordinates at every level
    if (c < ncomp && P->tile_w > 0 && ((TW % dx[c]) || (TH % dy[c]) || ((TW / dx[c]) % (1 << L)) ||
                                       ((TH / dy[c]) % (1 << L))))
      return -12;
  }
  const bool rev = P->reversible != 0;
  const bool same3 = ncomp >= 3 && dx[1] == dx[0] && dx[2] == dx[0] && dy[1] == dy[0] && dy[2] == dy[0];
  if (P->use_mct && ncomp >= 3 && !same3) return -12;  // the MCT needs equally sampled components
  const bool mct = P->use_mct && ncomp >= 3;
  const int mode =
      P->mode & (J2KENC_BYPASS | J2KENC_RESET | J2KENC_TERMALL | J2KENC_CAUSAL | J2KENC_PTERM | J2KENC_SEGSYM);
  int nthreads = P->num_threads > 0 ? P->num_threads : (int)std::thread::hardware_concurrency();
  if (nthreads < 1) nthreads = 1;
  const int ntx = ceil_div(W, TW), nty = ceil_div(H, TH);
  const int cbw = 1 << P->cbw_exp, cbh = 1 << P->cbh_exp;

  // synthesis energy gains per (level, low/high)
  std::vector<double> g_lo(L + 1, 1.0), g_hi(L + 1, 1.0);
  for (int l = 1; l <= L; ++l) {
    g_lo[l] = synth_gain_1d(rev, l, false);
    g_hi[l] = synth_gain_1d(rev, l, true);
  }

  // ---------------- tiles, transform, quantisation
  std::vector<Tile> tiles(ntx * nty);
  std::vector<int> band_eps_all, band_mu_all;  // QCD values (same for all tiles/components)
  int G = P->guard_bits > 0 ? P->guard_bits : (rev ? 2 : 1);
  // desired steps and QCD entries (computed once; identical for every tile-component)
  const int nbands_total = 3 * L + 1;
  std::vector<int> q_eps(nbands_total), q_mu(nbands_total), q_gain(nbands_total);
  std::vector<double> q_delta(nbands_total), q_w(nbands_total);
  for (int i = 0; i < nbands_total; ++i) {
    int lev, type;
    if (i == 0) {
      lev = L;
      type = 0;
    } else {
      lev = L - (i - 1) / 3;
      type = (i - 1) % 3 + 1;
    }
    int gain = (type == 0) ? 0 : (type == 3 ? 2 : 1);
    q_gain[i] = gain;
    double e = (L == 0) ? 1.0
                        : ((type & 1) ? g_hi[lev] : g_lo[lev]) * ((type & 2) ? g_hi[lev] : g_lo[lev]);
    if (L == 0) e = 1.0;
    int Rb = B + gain;
    if (rev) {
      q_eps[i] = Rb;
      q_mu[i] = 0;
      q_delta[i] = 1.0;
    } else {
      double bs = P->base_step > 0 ? P->base_step : 1.0 / 256.0;
      double delta = bs * std::ldexp(1.0, B) / std::sqrt(e);
      double u = delta / std::ldexp(1.0, Rb);
      int ex = (int)std::floor(std::log2(u));
      double m = u / std::ldexp(1.0, ex);
      int mu = (int)std::lround((m - 1.0) * 2048.0);
      int eps = -ex;
      if (mu >= 2048) {
        mu = 0;
        eps -= 1;
      }
      eps = std::max(0, std::min(31, eps));
      q_eps[i] = eps;
      q_mu[i] = mu;
      q_delta[i] = std::ldexp(1.0 + mu / 2048.0, Rb - eps);
    }
    q_w[i] = e * q_delta[i] * q_delta[i];
  }

  // per tile: transform and quantise
  struct QBand {
    std::vector<int32_t> q;
    int w, h;
  };
  std::vector<std::vector<std::vector<QBand>>> qb(tiles.size());  // [tile][comp][band index]
  int needG = G;
  for (int t = 0; t < (int)tiles.size(); ++t) {
    Tile &T = tiles[t];
    int tx = t % ntx, ty = t / ntx;
    T.x0 = tx * TW;
    T.y0 = ty * TH;
    T.x1 = std::min(W, T.x0 + TW);
    T.y1 = std::min(H, T.y0 + TH);
  }
  std::atomic<int> next_tile(0);
  std::vector<int> tile_needG(tiles.size(), 0);
  auto tile_worker = [&]() {
    std::vector<double> tmp, rowl, rowh, col, coll, colh;
    std::vector<int64_t> irow, il, ih;
    for (;;) {
      int t = next_tile.fetch_add(1);
      if (t >= (int)tiles.size()) break;
      Tile &T = tiles[t];
      // DC shift + MCT; component c covers [ceil(x0 / dx), ceil(x1 / dx)) of its own grid
      // (T.800 B.2-B.3), its sample (i, j) taken from the plane at (i * dx, j * dy)
      std::vector<std::vector<double>> cd(ncomp);
      std::vector<std::vector<int64_t>> ci(ncomp);
      int ctw[4], cth[4];
      for (int c = 0; c < ncomp; ++c) {
        const int cx0 = ceil_div(T.x0, dx[c]), cy0 = ceil_div(T.y0, dy[c]);
        ctw[c] = ceil_div(T.x1, dx[c]) - cx0;
        cth[c] = ceil_div(T.y1, dy[c]) - cy0;
        cd[c].resize((size_t)ctw[c] * cth[c]);
        ci[c].resize((size_t)ctw[c] * cth[c]);
        for (int y = 0; y < cth[c]; ++y)
          for (int x = 0; x < ctw[c]; ++x) {
            const size_t src = (size_t)(cy0 + y) * dy[c] * W + (size_t)(cx0 + x) * dx[c];
            int64_t v = (int64_t)planes[(size_t)c * W * H + src] - (1 << (B - 1));
            ci[c][(size_t)y * ctw[c] + x] = v;
            cd[c][(size_t)y * ctw[c] + x] = (double)v;
          }
      }
      if (mct) {
        const size_t np = (size_t)ctw[0] * cth[0];
        for (size_t i = 0; i < np; ++i) {
          if (rev) {
            int64_t r = ci[0][i], g = ci[1][i], b = ci[2][i];
            int64_t yv = r + 2 * g + b;
            ci[0][i] = yv >= 0 ? yv / 4 : -((-yv + 3) / 4);
            ci[1][i] = b - g;
            ci[2][i] = r - g;
          } else {
            double r = cd[0][i], g = cd[1][i], b = cd[2][i];
            cd[0][i] = 0.299 * r + 0.587 * g + 0.114 * b;
            cd[1][i] = -0.16875 * r - 0.33126 * g + 0.5 * b;
            cd[2][i] = 0.5 * r - 0.41869 * g - 0.08131 * b;
          }
        }
      }
      qb[t].resize(ncomp);
      for (int c = 0; c < ncomp; ++c) {
        // in-place Mallat decomposition over the tile-component
        const int tw = ctw[c], th = cth[c];
        int cw = tw, ch = th;
        std::vector<int64_t> &I = ci[c];
        std::vector<double> &D = cd[c];
        for (int l = 1; l <= L; ++l) {
          int nlw = (cw + 1) / 2, nlh = (ch + 1) / 2;
          // vertical first
          for (int x = 0; x < cw; ++x) {
            if (rev) {
              irow.resize(ch);
              il.resize(nlh);
              ih.resize(ch / 2 + 1);
              for (int y = 0; y < ch; ++y) irow[y] = I[(size_t)y * tw + x];
              fwd53(irow.data(), ch, il.data(), ih.data());
              for (int y = 0; y < nlh; ++y) I[(size_t)y * tw + x] = il[y];
              for (int y = 0; y < ch / 2; ++y) I[(size_t)(nlh + y) * tw + x] = ih[y];
            } else {
              col.resize(ch);
              coll.resize(nlh);
              colh.resize(ch / 2 + 1);
              for (int y = 0; y < ch; ++y) col[y] = D[(size_t)y * tw + x];
              fwd97(col.data(), ch, coll.data(), colh.data(), tmp);
              for (int y = 0; y < nlh; ++y) D[(size_t)y * tw + x] = coll[y];
              for (int y = 0; y < ch / 2; ++y) D[(size_t)(nlh + y) * tw + x] = colh[y];
            }
          }
          // then horizontal
          for (int y = 0; y < ch; ++y) {
            if (rev) {
              irow.assign(I.begin() + (size_t)y * tw, I.begin() + (size_t)y * tw + cw);
              il.resize(nlw);
              ih.resize(cw / 2 + 1);
              fwd53(irow.data(), cw, il.data(), ih.data());
              for (int x = 0; x < nlw; ++x) I[(size_t)y * tw + x] = il[x];
              for (int x = 0; x < cw / 2; ++x) I[(size_t)y * tw + nlw + x] = ih[x];
            } else {
              rowl.assign(D.begin() + (size_t)y * tw, D.begin() + (size_t)y * tw + cw);
              coll.resize(nlw);
              colh.resize(cw / 2 + 1);
              fwd97(rowl.data(), cw, coll.data(), colh.data(), tmp);
              for (int x = 0; x < nlw; ++x) D[(size_t)y * tw + x] = coll[x];
              for (int x = 0; x < cw / 2; ++x) D[(size_t)y * tw + nlw + x] = colh[x];
            }
          }
          cw = nlw;
          ch = nlh;
        }
        // extract bands: index 0 = LL_L, then (HL, LH, HH) for levels L..1
        qb[t][c].resize(nbands_total);
        int lw[12], lh[12];
        lw[0] = tw;
        lh[0] = th;
        for (int l = 1; l <= L; ++l) {
          lw[l] = (lw[l - 1] + 1) / 2;
          lh[l] = (lh[l - 1] + 1) / 2;
        }
        for (int bi = 0; bi < nbands_total; ++bi) {
          int lev, type;
          if (bi == 0) {
            lev = L;
            type = 0;
          } else {
            lev = L - (bi - 1) / 3;
            type = (bi - 1) % 3 + 1;
          }
          int ox = 0, oy = 0, bw, bh;
          if (type == 0) {
            bw = lw[lev];
            bh = lh[lev];
          } else {
            bw = (type & 1) ? lw[lev - 1] / 2 : lw[lev];
            bh = (type & 2) ? lh[lev - 1] / 2 : lh[lev];
            ox = (type & 1) ? lw[lev] : 0;
            oy = (type & 2) ? lh[lev] : 0;
          }
          QBand &Q = qb[t][c][bi];
          Q.w = bw;
          Q.h = bh;
          Q.q.assign((size_t)bw * bh, 0);
          int Mb = G + q_eps[bi] - 1;
          int32_t lim = Mb >= 31 ? 0x7FFFFFFF : (int32_t)((1u << Mb) - 1);
          int32_t maxq = 0;
          for (int y = 0; y < bh; ++y)
            for (int x = 0; x < bw; ++x) {
              size_t src = (size_t)(oy + y) * tw + ox + x;
              int64_t qv;
              if (rev) {
                qv = I[src];
              } else {
                double v = D[src] / q_delta[bi];
                qv = (int64_t)(v < 0 ? -std::floor(-v) : std::floor(v));
              }
              int32_t a = (int32_t)std::min<int64_t>(qv < 0 ? -qv : qv, 0x7FFFFFFF);
              maxq = std::max(maxq, a);
              if (!rev && a > lim) qv = qv < 0 ? -lim : lim;  // one guard bit: clamp
              Q.q[(size_t)y * bw + x] = (int32_t)qv;
            }
          if (rev) {
            int bits = maxq ? floor_log2((uint32_t)maxq) + 1 : 0;
            int need = bits - q_eps[bi] + 1;
            tile_needG[t] = std::max(tile_needG[t], need);
          }
        }
      }
    }
  };
  {
    std::vector<std::thread> th;
    int n = std::min<int>(nthreads, (int)tiles.size());
    for (int i = 0; i < n; ++i) th.emplace_back(tile_worker);
    for (auto &x : th) x.join();
  }
  if (rev)
    for (int v : tile_needG) needG = std::max(needG, v);
  G = std::min(7, needG);

  // ---------------- geometry: resolutions, bands, code-blocks (T.800 Annex B)
  for (int t = 0; t < (int)tiles.size(); ++t) {
    Tile &T = tiles[t];
    T.comps.resize(ncomp);
    for (int c = 0; c < ncomp; ++c) {
      TileComp &TC = T.comps[c];
      TC.x0 = ceil_div(T.x0, dx[c]);
      TC.y0 = ceil_div(T.y0, dy[c]);
      TC.x1 = ceil_div(T.x1, dx[c]);
      TC.y1 = ceil_div(T.y1, dy[c]);
      TC.res.resize(L + 1);
      for (int r = 0; r <= L; ++r) {
        Resolution &R = TC.res[r];
        int nb = L - r;
        R.x0 = ceil_div_pow2(TC.x0, nb);
        R.y0 = ceil_div_pow2(TC.y0, nb);
        R.x1 = ceil_div_pow2(TC.x1, nb);
        R.y1 = ceil_div_pow2(TC.y1, nb);
        int nbands = r == 0 ? 1 : 3;
        R.bands.resize(nbands);
        for (int b = 0; b < nbands; ++b) {
          Band &Bd = R.bands[b];
          Bd.type = r == 0 ? 0 : b + 1;
          int lev = r == 0 ? L : L - r + 1;
          int xob = Bd.type & 1, yob = (Bd.type >> 1) & 1;
          if (r == 0) {
            Bd.x0 = ceil_div_pow2(TC.x0, L);
            Bd.y0 = ceil_div_pow2(TC.y0, L);
            Bd.x1 = ceil_div_pow2(TC.x1, L);
            Bd.y1 = ceil_div_pow2(TC.y1, L);
          } else {
            int s = 1 << (lev - 1);
            Bd.x0 = ceil_div_pow2(TC.x0 - s * xob, lev);
            Bd.y0 = ceil_div_pow2(TC.y0 - s * yob, lev);
            Bd.x1 = ceil_div_pow2(TC.x1 - s * xob, lev);
            Bd.y1 = ceil_div_pow2(TC.y1 - s * yob, lev);
          }
          int bi = r == 0 ? 0 : 1 + (r - 1) * 3 + b;
          Bd.eps = q_eps[bi];
          Bd.mu = q_mu[bi];
          Bd.delta = q_delta[bi];
          Bd.weight = q_w[bi];
          Bd.Mb = G + q_eps[bi] - 1;
          int bw = Bd.x1 - Bd.x0, bh = Bd.y1 - Bd.y0;
          if (bw <= 0 || bh <= 0) {
            Bd.ncbx = Bd.ncby = 0;
            continue;
          }
          Bd.cbx0 = Bd.x0 / cbw;
          Bd.cby0 = Bd.y0 / cbh;
          Bd.ncbx = ceil_div(Bd.x1, cbw) - Bd.cbx0;
          Bd.ncby = ceil_div(Bd.y1, cbh) - Bd.cby0;
          Bd.cbs.resize((size_t)Bd.ncbx * Bd.ncby);
          for (int j = 0; j < Bd.ncby; ++j)
            for (int i = 0; i < Bd.ncbx; ++i) {
              CodeBlock &cb = Bd.cbs[(size_t)j * Bd.ncbx + i];
              int gx0 = std::max(Bd.x0, (Bd.cbx0 + i) * cbw), gx1 = std::min(Bd.x1, (Bd.cbx0 + i + 1) * cbw);
              int gy0 = std::max(Bd.y0, (Bd.cby0 + j) * cbh), gy1 = std::min(Bd.y1, (Bd.cby0 + j + 1) * cbh);
              cb.x0 = gx0 - Bd.x0;
              cb.y0 = gy0 - Bd.y0;
              cb.w = gx1 - gx0;
              cb.h = gy1 - gy0;
              cb.band = Bd.type;
            }
        }
      }
    }
  }

  // ---------------- Tier-1 (parallel over code-blocks)
  struct Job {
    int t, c, r, b, k;
  };
  std::vector<Job> jobs;
  for (int t = 0; t < (int)tiles.size(); ++t)
    for (int c = 0; c < ncomp; ++c)
      for (int r = 0; r <= L; ++r)
        for (int b = 0; b < (int)tiles[t].comps[c].res[r].bands.size(); ++b)
          for (int k = 0; k < (int)tiles[t].comps[c].res[r].bands[b].cbs.size(); ++k) jobs.push_back({t, c, r, b, k});
  std::atomic<size_t> next_job(0);
  auto t1_worker = [&]() {
    T1Coder coder;
    coder.mode = mode;
    for (;;) {
      size_t j = next_job.fetch_add(1);
      if (j >= jobs.size()) break;
      const Job &jb = jobs[j];
      Band &Bd = tiles[jb.t].comps[jb.c].res[jb.r].bands[jb.b];
      CodeBlock &cb = Bd.cbs[jb.k];
      int bi = jb.r == 0 ? 0 : 1 + (jb.r - 1) * 3 + jb.b;
      QBand &Q = qb[jb.t][jb.c][bi];
      coder.encode(Q.q.data() + (size_t)cb.y0 * Q.w + cb.x0, Q.w, cb, Bd.Mb, Bd.weight);
    }
  };
  {
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; ++i) th.emplace_back(t1_worker);
    for (auto &x : th) x.join();
  }
  qb.clear();

  // ---------------- layer formation (slope thresholds over per-pass rate/distortion)
  std::vector<CodeBlock *> all;
  for (auto &T : tiles)
    for (auto &TC : T.comps)
      for (auto &R : TC.res)
        for (auto &Bd : R.bands)
          for (auto &cb : Bd.cbs) all.push_back(&cb);
  const int NL = P->num_layers;
  for (CodeBlock *cb : all) cb->layer_passes.assign(NL, 0);
  // convex-hull truncation points per block
  std::vector<std::vector<int>> hull(all.size());
  std::vector<std::vector<double>> hull_slope(all.size());
  for (size_t i = 0; i < all.size(); ++i) {
    CodeBlock *cb = all[i];
    std::vector<int> &hp = hull[i];
    std::vector<double> &hs = hull_slope[i];
    double lastR = 0, lastD = 0;
    for (int k = 0; k < cb->npasses; ++k) {
      double R = cb->passes[k].end_len, D = cb->passes[k].dist;
      // pop points that are not on the convex hull
      for (;;) {
        double pr = hp.empty() ? 0 : cb->passes[hp.back()].end_len;
        double pd = hp.empty() ? 0 : cb->passes[hp.back()].dist;
        double dr = R - pr, dd = D - pd;
        double s = dr <= 0 ? (dd > 0 ? 1e300 : -1) : dd / dr;
        if (!hp.empty() && s >= hs.back()) {
          hp.pop_back();
          hs.pop_back();
          continue;
        }
        if (s > 0) {
          hp.push_back(k);
          hs.push_back(s);
        }
        break;
      }
      lastR = R;
      lastD = D;
    }
    (void)lastR;
    (void)lastD;
  }
  std::vector<int> prev(all.size(), 0);
  for (int l = 0; l < NL; ++l) {
    double bpp = P->layer_bpp[l];
    if (bpp <= 0) {
      for (size_t i = 0; i < all.size(); ++i) all[i]->layer_passes[l] = all[i]->npasses;
    } else {
      double budget = bpp * (double)W * H / 8.0;
      budget -= 64.0 * tiles.size() + 2.0 * all.size() * (l + 1) / 4.0;  // header estimate
      auto choose = [&](double lam, std::vector<int> &sel) -> double {
        double tot = 0;
        for (size_t i = 0; i < all.size(); ++i) {
          int n = prev[i];
          for (size_t h = 0; h < hull[i].size(); ++h)
            if (hull_slope[i][h] >= lam) n = std::max(n, hull[i][h] + 1);
          sel[i] = n;
          tot += n ? all[i]->passes[n - 1].end_len : 0;
        }
        return tot;
      };
      std::vector<int> sel(all.size());
      double lo = 0, hi = 1e30;
      // bisection in the log domain
      double llo = -60, lhi = 60;
      for (int it = 0; it < 60; ++it) {
        double mid = 0.5 * (llo + lhi);
        double tot = choose(std::exp2(mid), sel);
        if (tot > budget) llo = mid;
        else lhi = mid;
      }
      (void)lo;
      (void)hi;
      choose(std::exp2(lhi), sel);
      for (size_t i = 0; i < all.size(); ++i) all[i]->layer_passes[l] = sel[i];
    }
    for (size_t i = 0; i < all.size(); ++i) prev[i] = all[i]->layer_passes[l];
  }

  // ---------------- codestream
  const int markers = P->markers;
  const bool packed_hdrs = (markers & (J2KENC_PPM | J2KENC_PPT)) != 0;
  const int nparts = P->tile_parts > 1 ? P->tile_parts : 1;
  if ((markers & J2KENC_PPM) && (markers & J2KENC_PPT)) return -11;
  if (nparts > 255 || P->num_poc < 0 || P->num_poc > 8) return -11;
  for (int i = 0; i < P->num_poc; ++i) {
    const int *v = P->poc[i];
    if (v[0] < 0 || v[0] >= v[3] || v[3] > L + 1 || v[1] < 0 || v[1] >= v[4] || v[4] > ncomp || v[2] < 1 ||
        v[2] > NL || v[5] < 0 || v[5] > 4)
      return -11;
  }
  std::vector<uint8_t> cs;
  cs.reserve(1 << 20);
  put_u16(cs, 0xFF4F);  // SOC
  // SIZ
  put_u16(cs, 0xFF51);
  put_u16(cs, 38 + 3 * ncomp);
  put_u16(cs, 0);  // Rsiz
  put_u32(cs, W);
  put_u32(cs, H);
  put_u32(cs, 0);
  put_u32(cs, 0);
  put_u32(cs, TW);
  put_u32(cs, TH);
  put_u32(cs, 0);
  put_u32(cs, 0);
  put_u16(cs, ncomp);
  for (int c = 0; c < ncomp; ++c) {
    cs.push_back((uint8_t)(B - 1));
    cs.push_back((uint8_t)dx[c]);
    cs.push_back((uint8_t)dy[c]);
  }
  // COD
  put_u16(cs, 0xFF52);
  put_u16(cs, 12);
  cs.push_back((uint8_t)(((markers & J2KENC_SOP) ? 2 : 0) | ((markers & J2KENC_EPH) ? 4 : 0)));  // Scod
  cs.push_back((uint8_t)P->progression);
  put_u16(cs, NL);
  cs.push_back(mct ? 1 : 0);
  cs.push_back((uint8_t)L);
  cs.push_back((uint8_t)(P->cbw_exp - 2));
  cs.push_back((uint8_t)(P->cbh_exp - 2));
  cs.push_back((uint8_t)mode);
  cs.push_back(rev ? 1 : 0);
  // QCD
  put_u16(cs, 0xFF5C);
  if (rev) {
    put_u16(cs, 3 + nbands_total);
    cs.push_back((uint8_t)(G << 5));
    for (int i = 0; i < nbands_total; ++i) cs.push_back((uint8_t)(q_eps[i] << 3));
  } else {
    put_u16(cs, 3 + 2 * nbands_total);
    cs.push_back((uint8_t)((G << 5) | 2));
    for (int i = 0; i < nbands_total; ++i) put_u16(cs, (unsigned)((q_eps[i] << 11) | q_mu[i]));
  }
  // COM
  {
    const char msg[] = "j2k-b200 test encoder";
    put_u16(cs, 0xFF64);
    put_u16(cs, (unsigned)(4 + sizeof(msg) - 1));
    put_u16(cs, 1);
    cs.insert(cs.end(), msg, msg + sizeof(msg) - 1);
  }

  // tile-parts of every tile: header markers, body, and the packed packet headers (PPM / PPT)
  struct TilePart {
    std::vector<uint8_t> markers, body, packed;
  };
  std::vector<std::vector<TilePart>> tparts(tiles.size());
  for (int t = 0; t < (int)tiles.size(); ++t) {
    Tile &T = tiles[t];
    // reset T2 state
    for (auto &TC : T.comps)
      for (auto &R : TC.res)
        for (auto &Bd : R.bands)
          for (auto &cb : Bd.cbs) {
            cb.lblock = 3;
            cb.included = false;
          }
    // tag trees per (comp, res, band)
    std::vector<std::vector<std::vector<TagTree>>> incl(ncomp), zbp(ncomp);
    for (int c = 0; c < ncomp; ++c) {
      incl[c].resize(L + 1);
      zbp[c].resize(L + 1);
      for (int r = 0; r <= L; ++r) {
        auto &bands = T.comps[c].res[r].bands;
        incl[c][r].resize(bands.size());
        zbp[c][r].resize(bands.size());
        for (size_t b = 0; b < bands.size(); ++b) {
          Band &Bd = bands[b];
          if (Bd.cbs.empty()) continue;
          incl[c][r][b].build(Bd.ncbx, Bd.ncby);
          zbp[c][r][b].build(Bd.ncbx, Bd.ncby);
          std::vector<int> fl(Bd.cbs.size()), zb(Bd.cbs.size());
          for (size_t k = 0; k < Bd.cbs.size(); ++k) {
            CodeBlock &cb = Bd.cbs[k];
            int f = NL;
            for (int l = 0; l < NL; ++l)
              if (cb.layer_passes[l] > 0) {
                f = l;
                break;
              }
            fl[k] = f;
            zb[k] = cb.missing;
          }
          incl[c][r][b].set_values(fl);
          zbp[c][r][b].set_values(zb);
        }
      }
    }
    struct Packet {
      std::vector<uint8_t> hdr, body;
    };
    std::vector<Packet> pkts;
    auto emit_packet = [&](int l, int r, int c) {
      Resolution &R = T.comps[c].res[r];
      if (R.x1 <= R.x0 || R.y1 <= R.y0) return;  // no precinct
      std::vector<uint8_t> hdr;
      BitWriter bw(hdr);
      bool any = false;
      for (auto &Bd : R.bands)
        for (auto &cb : Bd.cbs) {
          int before = l ? cb.layer_passes[l - 1] : 0;
          if (cb.layer_passes[l] > before) any = true;
        }
      std::vector<std::pair<const uint8_t *, size_t>> pieces;
      if (!any) {
        bw.put(0);
      } else {
        bw.put(1);
        for (size_t b = 0; b < R.bands.size(); ++b) {
          Band &Bd = R.bands[b];
          for (size_t k = 0; k < Bd.cbs.size(); ++k) {
            CodeBlock &cb = Bd.cbs[k];
            int before = l ? cb.layer_passes[l - 1] : 0;
            int nnew = cb.layer_passes[l] - before;
            if (!cb.included) {
              incl[c][r][b].encode(bw, (int)k, l + 1);
            } else {
              bw.put(nnew > 0);
            }
            if (nnew <= 0) continue;
            if (!cb.included) {
              zbp[c][r][b].encode(bw, (int)k, 1 << 20);
              cb.included = true;
            }
            // number of passes
            if (nnew == 1) bw.put(0);
            else if (nnew == 2) bw.put_bits(2, 2);
            else if (nnew <= 5) bw.put_bits(0xC | (nnew - 3), 4);
            else if (nnew <= 36) bw.put_bits((0xF << 5) | (nnew - 6), 9);
            else bw.put_bits((0x1FFu << 7) | (unsigned)(nnew - 37), 16);
            // segment pieces of this contribution
            std::vector<std::pair<int, uint32_t>> seg;  // (passes, bytes)
            int s = before;
            while (s < before + nnew) {
              int e = s + 1;
              while (e < before + nnew && !seg_starts(mode, e)) ++e;
              uint32_t b0 = s ? cb.passes[s - 1].end_len : 0;
              // pass s may be in the middle of a segment whose earlier passes were in
              // an earlier layer; bytes counted from the previous pass end
              uint32_t b1 = cb.passes[e - 1].end_len;
              seg.push_back({e - s, b1 - b0});
              s = e;
            }
            int inc = 0;
            for (auto &sg : seg) {
              int bits = cb.lblock + floor_log2((uint32_t)sg.first);
              while ((int64_t)sg.second >= ((int64_t)1 << (bits + inc))) ++inc;
            }
            for (int i = 0; i < inc; ++i) bw.put(1);
            bw.put(0);
            cb.lblock += inc;
            for (auto &sg : seg) bw.put_bits(sg.second, cb.lblock + floor_log2((uint32_t)sg.first));
            uint32_t b0 = before ? cb.passes[before - 1].end_len : 0;
            uint32_t b1 = cb.passes[before + nnew - 1].end_len;
            pieces.push_back({cb.data.data() + b0, (size_t)(b1 - b0)});
          }
        }
      }
      bw.flush();
      Packet pk;
      pk.hdr = std::move(hdr);
      for (auto &pc : pieces) pk.body.insert(pk.body.end(), pc.first, pc.first + pc.second);
      pkts.push_back(std::move(pk));
    };
    // packet order: the progression volumes, each packet once (T.800 B.12)
    std::vector<std::vector<int>> next_layer(ncomp, std::vector<int>(L + 1, 0));
    auto visit = [&](int l, int r, int c) {
      if (next_layer[c][r] != l) return;
      next_layer[c][r] = l + 1;
      emit_packet(l, r, c);
    };
    std::vector<std::vector<int>> vols;
    for (int i = 0; i < P->num_poc; ++i) vols.push_back(std::vector<int>(P->poc[i], P->poc[i] + 6));
    if (vols.empty()) vols.push_back({0, 0, NL, L + 1, ncomp, P->progression});
    for (auto &v : vols) {
      const int rs = v[0], c0 = v[1], lye = v[2], re = v[3], ce = v[4];
      switch (v[5]) {
        case J2KENC_LRCP:
          for (int l = 0; l < lye; ++l)
            for (int r = rs; r < re; ++r)
              for (int c = c0; c < ce; ++c) visit(l, r, c);
          break;
        case J2KENC_RLCP:
          for (int r = rs; r < re; ++r)
            for (int l = 0; l < lye; ++l)
              for (int c = c0; c < ce; ++c) visit(l, r, c);
          break;
        case J2KENC_RPCL:
          for (int r = rs; r < re; ++r)
            for (int c = c0; c < ce; ++c)
              for (int l = 0; l < lye; ++l) visit(l, r, c);
          break;
        default:  // PCRL, CPRL: one precinct per resolution, all at the tile origin
          for (int c = c0; c < ce; ++c)
            for (int r = rs; r < re; ++r)
              for (int l = 0; l < lye; ++l) visit(l, r, c);
          break;
      }
    }
    for (int c = 0; c < ncomp; ++c)
      for (int r = 0; r <= L; ++r)
        if (next_layer[c][r] != NL) return -10;  // the volumes leave packets out
    // tile-parts: SOP before each packet, EPH after each header, headers packed or inline
    const size_t n = pkts.size();
    int zppt = 0;
    for (int k = 0; k < nparts; ++k) {
      TilePart tp;
      for (size_t i = k * n / nparts; i < (k + 1) * n / nparts; ++i) {
        if (markers & J2KENC_SOP) {
          put_u16(tp.body, 0xFF91);
          put_u16(tp.body, 4);
          put_u16(tp.body, (unsigned)(i & 0xFFFF));
        }
        std::vector<uint8_t> &h = packed_hdrs ? tp.packed : tp.body;
        h.insert(h.end(), pkts[i].hdr.begin(), pkts[i].hdr.end());
        if (markers & J2KENC_EPH) put_u16(h, 0xFF92);
        tp.body.insert(tp.body.end(), pkts[i].body.begin(), pkts[i].body.end());
      }
      if (k == 0 && P->num_poc && P->poc_in_tiles) {
        put_u16(tp.markers, 0xFF5F);
        put_u16(tp.markers, (unsigned)(2 + 7 * P->num_poc));
        for (int i = 0; i < P->num_poc; ++i) {
          const int *v = P->poc[i];
          tp.markers.push_back((uint8_t)v[0]);
          tp.markers.push_back((uint8_t)v[1]);
          put_u16(tp.markers, (unsigned)v[2]);
          tp.markers.push_back((uint8_t)v[3]);
          tp.markers.push_back((uint8_t)v[4]);
          tp.markers.push_back((uint8_t)v[5]);
        }
      }
      if (markers & J2KENC_PPT) {  // PPT segments of at most 65532 header bytes
        size_t off = 0;
        do {
          const size_t m = std::min<size_t>(65532, tp.packed.size() - off);
          if (zppt > 255) return -12;
          put_u16(tp.markers, 0xFF61);
          put_u16(tp.markers, (unsigned)(3 + m));
          tp.markers.push_back((uint8_t)zppt++);
          tp.markers.insert(tp.markers.end(), tp.packed.begin() + off, tp.packed.begin() + off + m);
          off += m;
        } while (off < tp.packed.size());
      }
      tparts[t].push_back(std::move(tp));
    }
  }
  // codestream order of the tile-parts
  std::vector<std::pair<int, int>> order;
  if (P->interleave_tile_parts) {
    for (int k = 0; k < nparts; ++k)
      for (int t = 0; t < (int)tiles.size(); ++t) order.push_back({t, k});
  } else {
    for (int t = 0; t < (int)tiles.size(); ++t)
      for (int k = 0; k < nparts; ++k) order.push_back({t, k});
  }
  if (P->num_poc && !P->poc_in_tiles) {  // main-header POC
    put_u16(cs, 0xFF5F);
    put_u16(cs, (unsigned)(2 + 7 * P->num_poc));
    for (int i = 0; i < P->num_poc; ++i) {
      const int *v = P->poc[i];
      cs.push_back((uint8_t)v[0]);
      cs.push_back((uint8_t)v[1]);
      put_u16(cs, (unsigned)v[2]);
      cs.push_back((uint8_t)v[3]);
      cs.push_back((uint8_t)v[4]);
      cs.push_back((uint8_t)v[5]);
    }
  }
  if (markers & J2KENC_PPM) {  // Nppm + headers of every tile-part, in codestream order
    std::vector<uint8_t> ppm;
    for (auto &o : order) {
      const TilePart &tp = tparts[o.first][o.second];
      put_u32(ppm, (uint32_t)tp.packed.size());
      ppm.insert(ppm.end(), tp.packed.begin(), tp.packed.end());
    }
    size_t off = 0;
    for (int z = 0; off < ppm.size(); ++z) {
      if (z > 255) return -12;
      const size_t m = std::min<size_t>(65532, ppm.size() - off);
      put_u16(cs, 0xFF60);
      put_u16(cs, (unsigned)(3 + m));
      cs.push_back((uint8_t)z);
      cs.insert(cs.end(), ppm.begin() + off, ppm.begin() + off + m);
      off += m;
    }
  }
  for (auto &o : order) {  // SOT + tile-part header markers + SOD + body
    const TilePart &tp = tparts[o.first][o.second];
    put_u16(cs, 0xFF90);
    put_u16(cs, 10);
    put_u16(cs, (unsigned)o.first);
    put_u32(cs, (uint32_t)(12 + tp.markers.size() + 2 + tp.body.size()));
    cs.push_back((uint8_t)o.second);
    cs.push_back((uint8_t)nparts);
    cs.insert(cs.end(), tp.markers.begin(), tp.markers.end());
    put_u16(cs, 0xFF93);
    cs.insert(cs.end(), tp.body.begin(), tp.body.end());
  }
  put_u16(cs, 0xFFD9);  // EOC
  *out = (uint8_t *)std::malloc(cs.size());
  if (!*out) return -9;
  std::memcpy(*out, cs.data(), cs.size());
  *out_len = cs.size();
  return 0;
}
