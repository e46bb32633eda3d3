/*
 * codestream.cpp — host-side JPEG 2000 Part-1 front end (markers, tiles, Tier-2).
 *
 * Produces the flat decode plan of plan.h.  Follows ITU-T T.800 Annex A (markers) and
 * Annex B (geometry, tag trees, packet headers).  Reference counterparts:
 * decoder/codec/src/dec_syntax.cpp:134-421 (main/tile headers), dec_packet.cpp:66-221
 * (packet header: inclusion, zero bit-planes, pass count, Lblock, lengths) and :384-730
 * (progression orders), dec_init.cpp:645-1056 (tile/subband/code-block geometry),
 * dec_jp2.cpp:46-66,466-523 (supported-stream limits).
 *
 * Differences from the reference front end, by design: codeword segments are tracked per
 * code-block (the reference treats the whole pass list as one segment,
 * bmi_block_decoder.cpp:735-768), so BYPASS/RESET/TERMALL streams are planned correctly;
 * the 9/7 magnitude bit count is exponent + guard bits - 1 (T.800 E.1.1.1) where the
 * reference adds the guard bits to the raw exponent/mantissa word (dec_jp2.cpp:177-178),
 * which agrees only for one guard bit.
 */
#include "codestream.h"

#include <algorithm>
#include <atomic>
#include <exception>
#include <memory>
#include <mutex>
#include <thread>
#include <cstring>

namespace j2k {
namespace {

inline int ceil_div_pow2(int a, int l) { return (int)(((int64_t)a + (1LL << l) - 1) >> l); }
inline int ceil_div(int a, int b) { return (int)(((int64_t)a + b - 1) / b); }
inline int floor_log2(uint32_t v) { return v ? 31 - __builtin_clz(v) : -1; }

struct Reader {
  const uint8_t *p, *end;
  bool ok = true;
  size_t left() const { return (size_t)(end - p); }
  unsigned u8() {
    if (p >= end) {
      ok = false;
      return 0;
    }
    return *p++;
  }
  unsigned u16() {
    unsigned a = u8();
    return (a << 8) | u8();
  }
  uint32_t u32() {
    uint32_t a = u16();
    return (a << 16) | u16();
  }
};

// packet-header bit reader with 0xFF bit stuffing (T.800 B.10.1): after a 0xFF byte the
// next byte carries 7 bits (its most significant bit is a stuffed 0).  Bits are buffered in
// a 64-bit accumulator a byte at a time, so multi-bit fields are read in one step.
struct BitReader {
  const uint8_t *p, *end;
  uint32_t c = 0;     // the last byte read (0xFF decides the next byte's width)
  uint64_t acc = 0;   // unread bits, right-aligned
  int nacc = 0;       // number of unread bits
  bool overrun = false;
  void refill() {
    const uint32_t prev = c;
    if (p >= end) {
      overrun = true;
      c = 0;
    } else {
      c = *p++;
    }
    const int nb = (prev == 0xFF) ? 7 : 8;
    acc = (acc << nb) | (c & ((1u << nb) - 1u));
    nacc += nb;
  }
  int bit() {
    if (nacc == 0) refill();
    --nacc;
    return (int)((acc >> nacc) & 1);
  }
  uint32_t bits(int n) {
    while (nacc < n) refill();
    nacc -= n;
    return (uint32_t)((acc >> nacc) & ((n >= 32) ? 0xFFFFFFFFull : ((1ull << n) - 1)));
  }
  // end of header: byte aligned, a byte after 0xFF is consumed as well
  void align() {
    if (c == 0xFF && p < end) ++p;  // a header ending on 0xFF is followed by a stuffed byte
    nacc = 0;
    acc = 0;
    c = 0;
  }
};

struct TagTree {
  struct Node {
    int value, low, parent;
  };
  std::vector<Node> nodes;
  void build(int w, int h) {
    nodes.clear();
    if (w <= 0 || h <= 0) return;
    // level sizes halve up to a single root: at most 32 levels for 31-bit sizes
    int dw[34], dh[34], base[34], nl = 0, total = 0;
    dw[0] = w;
    dh[0] = h;
    for (;;) {
      base[nl] = total;
      total += dw[nl] * dh[nl];
      if (dw[nl] == 1 && dh[nl] == 1) break;
      dw[nl + 1] = (dw[nl] + 1) / 2;
      dh[nl + 1] = (dh[nl] + 1) / 2;
      ++nl;
    }
    nodes.assign(total, {1 << 30, 0, -1});
    for (int l = 0; l < nl; ++l)
      for (int y = 0; y < dh[l]; ++y)
        for (int x = 0; x < dw[l]; ++x) nodes[base[l] + y * dw[l] + x].parent = base[l + 1] + (y / 2) * dw[l + 1] + x / 2;
  }
  // returns 1 when the leaf value is below `threshold` (T.800 B.10.2)
  int decode(BitReader &br, int leaf, int threshold) {
    int stk[40], sp = 0, node = leaf;
    while (nodes[node].parent >= 0) {
      stk[sp++] = node;
      node = nodes[node].parent;
    }
    int low = 0;
    for (;;) {
      Node &n = nodes[node];
      if (low > n.low) n.low = low;
      else low = n.low;
      while (low < threshold && low < n.value) {
        if (br.bit()) n.value = low;
        else ++low;
        if (br.overrun) return 0;
      }
      n.low = low;
      if (!sp) break;
      node = stk[--sp];
    }
    return nodes[leaf].value < threshold ? 1 : 0;
  }
};

// A block's coded pieces (one per contributing layer and segment) and codeword-segment
// lengths are singly linked lists in per-tile arrays, so blocks allocate nothing.
struct Piece {
  const uint8_t *p;
  uint32_t len;
  int32_t next;
};
struct SegLen {
  uint32_t len;
  int32_t next;
};

struct CbState {
  int x0, y0, w, h;        // band coordinates relative to the band origin
  int passes = 0;          // passes signalled so far
  int kept = 0;            // passes of the layers being decoded
  int lblock = 3;
  int missing = 0;
  bool included = false;
  int32_t piece_head = -1, piece_tail = -1;  // into the tile's Piece array
  int32_t seg_head = -1, seg_tail = -1;      // into the tile's SegLen array
  uint32_t nseg = 0;                         // codeword segments
};

struct BandState {
  int type;                 // 0 LL 1 HL 2 LH 3 HH
  int x0, y0, x1, y1;       // absolute band coordinates
  int cbw_exp, cbh_exp;     // code-block size exponents (limited by precincts)
  uint16_t spqcd;
  int mb;                   // ref numbps (see plan.h)
  float gain;
  int off_x, off_y;         // position inside the tile-component Mallat region
  // code-blocks grouped by precinct
  std::vector<std::vector<int>> prec_cbs;   // [precinct] -> indices into cbs
  std::vector<TagTree> incl, zbp;
  std::vector<CbState> cbs;
};

struct ResState {
  int x0, y0, x1, y1;
  int npx = 0, npy = 0;     // precinct grid
  std::vector<BandState> bands;
};

struct TCState {
  int x0, y0, x1, y1;
  int levels;
  int comp;
  std::vector<ResState> res;
  uint64_t coef_off = 0;
};

// The coded bytes of a plan are the concatenation of spans (pointer into the codestream,
// length), cut into chunks of about 1 MB; a plan of at least 4 MB copies its chunks on up
// to 8 threads.
struct CopyChunk {
  uint8_t *dst;
  const std::pair<const uint8_t *, uint32_t> *b, *e;
};
void copy_chunks(const std::vector<CopyChunk> &chunks, size_t total) {
  auto run = [&](const CopyChunk &k) {
    uint8_t *o = k.dst;
    for (auto *sp = k.b; sp != k.e; ++sp) {
      std::memcpy(o, sp->first, sp->second);
      o += sp->second;
    }
  };
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = total >= (size_t(4) << 20) ? std::min<size_t>(std::min<size_t>(8, hw), chunks.size()) : 1;
  if (nt <= 1) {
    for (const CopyChunk &k : chunks) run(k);
    return;
  }
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    for (size_t i; (i = next.fetch_add(1)) < chunks.size();) run(chunks[i]);
  };
  std::vector<std::thread> th;
  for (size_t i = 1; i < nt; ++i) {
    try {
      th.emplace_back(worker);
    } catch (...) {  // no thread: the others take its share
      break;
    }
  }
  worker();
  for (auto &x : th) x.join();
}

// First pass after pass s that starts a new codeword segment (T.800 D.4.1 and D.6): every
// pass with TERMALL; with BYPASS, passes 0-9 share the first (MQ) segment and later ones
// alternate a raw segment (significance + refinement) and an MQ one (cleanup); otherwise no
// later segment
int next_seg_start(int style, int s) {
  if (style & J2K_CB_TERMALL) return s + 1;
  if (!(style & J2K_CB_BYPASS)) return 1 << 30;
  if (s < 10) return 10;
  return ((s - 1) % 3 == 0) ? s + 2 : s + 1;
}

bool seg_starts(int style, int j) {
  int type = (j == 0) ? 2 : (j - 1) % 3;
  if (j == 0) return true;
  if (style & J2K_CB_TERMALL) return true;
  return (style & J2K_CB_BYPASS) && j >= 10 && type != 1;
}

}  // namespace

const char *status_string(int s) {
  switch (s) {
    case PARSE_OK: return "ok";
    case PARSE_ERR_TRUNCATED: return "truncated codestream";
    case PARSE_ERR_MARKER: return "bad marker";
    case PARSE_ERR_UNSUPPORTED: return "unsupported feature";
    case PARSE_ERR_INVALID: return "invalid parameter";
    case PARSE_ERR_PACKET: return "corrupt packet";
    default: return "unknown";
  }
}

float irrev_band_gain(uint16_t spqcd, int bitdepth, int band, int no_dwt) {
  // Delta' as in bmi_cpu_dwt_decoder.cpp:1035-1044 (integer shift, then * 2^-13), and the
  // separable K gains of :1433-1473 (horizontal factor, then vertical factor).
  int abs_step = ((spqcd & 0x7ff) << 2) | 0x2000;
  int n = bitdepth - (spqcd >> 11);
  abs_step = (n > 0) ? (abs_step << n) : (abs_step >> (-n));
  volatile float norm = (float)abs_step * 0.0001220703125f;
  const float klo = 1.23017410558578f, khi = 1.62578613134411f;
  volatile float g;
  if (no_dwt) return norm;  // no lifting stage to fold the K gains into
  switch (band) {
    case 0: g = norm * klo; g = g * klo; break;
    case 1: g = norm * khi; g = g * klo; break;
    case 2: g = norm * klo; g = g * khi; break;
    default: g = norm * khi; g = g * khi; break;
  }
  return g;
}

float irrev_ll_gain() {
  volatile float klo = 1.23017410558578f;
  volatile float g = klo * klo;
  return g;
}

// JP2 file format (T.800 Annex I): walk the boxes to the contiguous codestream box 'jp2c',
// reading the colour specification of the header box on the way.  Mirrors the reference's
// dec_read_jp2_header (dec_syntax.cpp:38-133): the signature and file-type boxes come first,
// the header box (with ihdr / bpcc / colr / pclr / cmap / cdef / res) before 'jp2c', and the
// colour specification's method and enumerated colour space are kept.  Unlike the reference,
// boxes it does not know are skipped rather than refused (T.800 I.4).  Returns the offset of
// the codestream, 0 for a bare codestream, (size_t)-1 for a malformed wrapper.
static size_t find_codestream(const uint8_t *d, size_t len, StreamHeader &H) {
  if (!(len >= 12 && d[0] == 0 && d[1] == 0 && d[2] == 0 && d[3] == 12 && d[4] == 'j' && d[5] == 'P')) return 0;
  auto be32 = [&](size_t at) -> uint32_t {
    return ((uint32_t)d[at] << 24) | ((uint32_t)d[at + 1] << 16) | ((uint32_t)d[at + 2] << 8) | d[at + 3];
  };
  // one box header at `pos` of [pos, limit): content start and end
  auto box = [&](size_t pos, size_t limit, uint32_t &type, size_t &body, size_t &next) -> bool {
    if (pos + 8 > limit) return false;
    uint64_t lbox = be32(pos);
    type = be32(pos + 4);
    size_t hdr = 8;
    if (lbox == 1) {
      if (pos + 16 > limit) return false;
      lbox = ((uint64_t)be32(pos + 8) << 32) | be32(pos + 12);
      hdr = 16;
    } else if (lbox == 0) {
      lbox = limit - pos;
    }
    if (lbox < hdr || lbox > limit - pos) return false;
    body = pos + hdr;
    next = pos + (size_t)lbox;
    return true;
  };
  bool ftyp = false, jp2h = false;
  size_t pos = 0;
  for (;;) {
    uint32_t type;
    size_t body, next;
    if (!box(pos, len, type, body, next)) return (size_t)-1;
    if (type == 0x6A703263) return jp2h ? body : (size_t)-1;  // 'jp2c' after the header box
    if (type == 0x66747970) ftyp = true;                       // 'ftyp'
    if (type == 0x6A703268) {                                  // 'jp2h'
      if (!ftyp) return (size_t)-1;
      for (size_t q = body; q < next;) {
        uint32_t st;
        size_t sb, sn;
        if (!box(q, next, st, sb, sn)) return (size_t)-1;
        if (st == 0x636F6C72 && sn - sb >= 3 && !H.jp2_colr_method) {  // 'colr': the first one counts
          H.jp2_colr_method = d[sb];
          if (d[sb] == 1 && sn - sb >= 7) H.jp2_colr_enum = (int)be32(sb + 3);
        }
        q = sn;
      }
      jp2h = true;
    }
    pos = next;
  }
}

namespace {

// SPcod / SPcoc of one component (T.800 Table A.15): levels, code-block size and style,
// transform, precinct sizes
int read_spcod(Reader &s, StreamHeader &H, int c, bool user_precincts) {
  const int lev = (int)s.u8();
  const int xcb = (int)s.u8() + 2, ycb = (int)s.u8() + 2;
  const int style = (int)s.u8();
  const int rev = s.u8() == 1;
  if (lev > J2K_MAX_LEVELS) return PARSE_ERR_UNSUPPORTED;
  H.levels[c] = lev;
  H.cbw_exp[c] = xcb;
  H.cbh_exp[c] = ycb;
  H.cbstyle[c] = style;
  H.reversible[c] = rev;
  for (int i = 0; i <= lev; ++i) {
    if (user_precincts) {
      unsigned pp = s.u8();
      H.ppx[c][i] = pp & 0xF;
      H.ppy[c][i] = pp >> 4;
      if (i > 0 && (H.ppx[c][i] == 0 || H.ppy[c][i] == 0)) return PARSE_ERR_INVALID;
    } else {
      H.ppx[c][i] = H.ppy[c][i] = 15;
    }
  }
  return s.ok ? PARSE_OK : PARSE_ERR_TRUNCATED;
}

// COD (A.6.1): the image- or tile-wide SGcod, and SPcod for every component that no COC of
// equal or higher precedence has set (`comp_set`)
int read_cod(Reader s, StreamHeader &H, const bool *comp_set) {
  const unsigned scod = s.u8();
  H.progression = (int)s.u8();
  H.layers = (int)s.u16();
  H.mct = (int)s.u8();
  H.sop = (scod >> 1) & 1;
  H.eph = (scod >> 2) & 1;
  if (!s.ok) return PARSE_ERR_TRUNCATED;
  if (H.progression > 4) return PARSE_ERR_INVALID;
  for (int c = 0; c < J2K_MAX_COMPONENTS; ++c) {
    if (comp_set[c]) continue;
    Reader t = s;
    const int rc = read_spcod(t, H, c, scod & 1);
    if (rc != PARSE_OK) return rc;
  }
  return PARSE_OK;
}

// COC (A.6.2)
int read_coc(Reader s, StreamHeader &H, bool *comp_set) {
  const int c = H.ncomp < 257 ? (int)s.u8() : (int)s.u16();
  if (c >= H.ncomp) return PARSE_ERR_INVALID;
  const unsigned scoc = s.u8();
  const int rc = read_spcod(s, H, c, scoc & 1);
  comp_set[c] = true;
  return rc;
}

// QCD / QCC (A.6.4, A.6.5); a QCD leaves the components that a QCC of equal or higher
// precedence has set (`comp_set`)
int read_qcx(Reader s, bool qcc, StreamHeader &H, bool *comp_set) {
  int c0 = 0, c1 = J2K_MAX_COMPONENTS;
  if (qcc) {
    c0 = H.ncomp < 257 ? (int)s.u8() : (int)s.u16();
    if (c0 >= H.ncomp) return PARSE_ERR_INVALID;
    c1 = c0 + 1;
  }
  const unsigned sq = s.u8();
  const int style = sq & 0x1F, guard = (int)(sq >> 5);
  std::vector<uint16_t> st;
  while (s.left() > 0) {
    if (style == 0) st.push_back((uint16_t)(s.u8() >> 3));
    else st.push_back((uint16_t)s.u16());
  }
  if (!s.ok) return PARSE_ERR_TRUNCATED;
  if (style > 2 || (style == 1 && st.size() != 1)) return PARSE_ERR_INVALID;
  if (st.empty() || st.size() > 3 * J2K_MAX_LEVELS + 1) return PARSE_ERR_INVALID;
  for (int c = c0; c < c1; ++c) {
    if (!qcc && comp_set[c]) continue;
    H.qstyle[c] = style;
    H.guard[c] = guard;
    for (size_t i = 0; i < 3 * J2K_MAX_LEVELS + 1; ++i) H.steps[c][i] = i < st.size() ? st[i] : 0;
    if (qcc) comp_set[c] = true;
  }
  return PARSE_OK;
}

// RGN (A.6.3): only the shift is kept (a non-zero shift is refused later)
int read_rgn(Reader s, StreamHeader &H) {
  const int c = H.ncomp < 257 ? (int)s.u8() : (int)s.u16();
  s.u8();
  const int shift = (int)s.u8();
  if (!s.ok) return PARSE_ERR_TRUNCATED;
  if (c < J2K_MAX_COMPONENTS) H.roi_shift[c] = shift;
  return PARSE_OK;
}

// POC (A.6.6): progression volumes appended to `out`; CEpoc 0 stands for 256 (8-bit form)
int read_poc(Reader s, int ncomp, std::vector<PocEntry> &out) {
  const bool wide = ncomp >= 257;
  const size_t entry = wide ? 9 : 7;
  if (s.left() == 0 || s.left() % entry) return PARSE_ERR_INVALID;
  while (s.left() >= entry) {
    PocEntry e;
    e.rs = (int)s.u8();
    e.cs = wide ? (int)s.u16() : (int)s.u8();
    e.lye = (int)s.u16();
    e.re = (int)s.u8();
    e.ce = wide ? (int)s.u16() : (int)s.u8();
    if (!wide && e.ce == 0) e.ce = 256;
    e.prog = (int)s.u8();
    if (e.prog > 4) return PARSE_ERR_INVALID;
    out.push_back(e);
  }
  return PARSE_OK;
}

// checks of the coding parameters against what the plan and the device path support, and
// the expansion of scalar-derived quantisation (T.800 E.1.1.1); `main` is the main header
// when H is a tile's parameters
int finish_coding(StreamHeader &H, const StreamHeader *main) {
  if (H.layers < 1) return PARSE_ERR_INVALID;
  for (int c = 0; c < H.ncomp; ++c) {
    if (H.cbw_exp[c] > 10 || H.cbh_exp[c] > 10 || H.cbw_exp[c] + H.cbh_exp[c] > 12) return PARSE_ERR_INVALID;
    if (H.cbw_exp[c] > 6 || H.cbh_exp[c] > 6) return PARSE_ERR_UNSUPPORTED;  // device kernels: <= 64
    if (H.roi_shift[c]) return PARSE_ERR_UNSUPPORTED;
    // the device runs one wavelet and one inverse MCT per image
    if (H.reversible[c] != H.reversible[0]) return PARSE_ERR_UNSUPPORTED;
    if (H.qstyle[c] == 1) {  // scalar derived: expand to the expounded form
      uint16_t b = H.steps[c][0];
      int eps0 = b >> 11, mu0 = b & 0x7FF;
      for (int i = 1; i <= 3 * H.levels[c]; ++i) {
        int nb = H.levels[c] - (i - 1) / 3;
        int eps = eps0 - H.levels[c] + nb;
        H.steps[c][i] = (uint16_t)(((eps < 0 ? 0 : eps) << 11) | mu0);
      }
    }
  }
  if (main && (H.reversible[0] != main->reversible[0] || H.mct != main->mct)) return PARSE_ERR_UNSUPPORTED;
  // the inverse RCT / ICT combines the first three components sample by sample, which needs
  // them sampled alike (T.800 G.1)
  if (H.mct && H.ncomp >= 3)
    for (int c = 1; c < 3; ++c)
      if (H.sub_x[c] != H.sub_x[0] || H.sub_y[c] != H.sub_y[0]) return PARSE_ERR_UNSUPPORTED;
  return PARSE_OK;
}

}  // namespace

int parse_header(const uint8_t *data, size_t len, StreamHeader &H) {
  H = StreamHeader();
  size_t off = find_codestream(data, len, H);
  if (off == (size_t)-1) return PARSE_ERR_MARKER;
  // an enumerated colour space other than sRGB, greyscale or sYCC is refused, as the
  // reference refuses it (dec_jp2.cpp:462-464)
  if (H.jp2_colr_method == 1 && H.jp2_colr_enum != 16 && H.jp2_colr_enum != 17 && H.jp2_colr_enum != 18)
    return PARSE_ERR_UNSUPPORTED;
  H.cs_offset = off;
  Reader r{data + off, data + len};
  if (r.u16() != 0xFF4F) return PARSE_ERR_MARKER;
  bool have_siz = false, have_cod = false, have_qcd = false;
  bool coc_set[J2K_MAX_COMPONENTS] = {false}, qcc_set[J2K_MAX_COMPONENTS] = {false};
  std::vector<std::pair<int, std::pair<const uint8_t *, size_t>>> ppm;  // (Zppm, payload)
  for (;;) {
    if (r.left() < 4) return PARSE_ERR_TRUNCATED;
    unsigned m = r.u16();
    if (m == 0xFF90) {
      r.p -= 2;
      break;
    }
    if (m < 0xFF30) return PARSE_ERR_MARKER;
    unsigned lseg = r.u16();
    if (lseg < 2 || lseg - 2 > r.left()) return PARSE_ERR_TRUNCATED;
    Reader s{r.p, r.p + (lseg - 2)};
    r.p += lseg - 2;
    int rc = PARSE_OK;
    if (m != 0xFF51 && m != 0xFF64 && !have_siz) return PARSE_ERR_MARKER;  // SIZ comes first
    switch (m) {
      case 0xFF51: {  // SIZ
        s.u16();
        H.width = (int)s.u32();
        H.height = (int)s.u32();
        H.x0 = (int)s.u32();
        H.y0 = (int)s.u32();
        H.tile_w = (int)s.u32();
        H.tile_h = (int)s.u32();
        H.tx0 = (int)s.u32();
        H.ty0 = (int)s.u32();
        H.ncomp = (int)s.u16();
        if (H.ncomp < 1 || H.ncomp > J2K_MAX_COMPONENTS) return PARSE_ERR_UNSUPPORTED;
        for (int c = 0; c < H.ncomp; ++c) {
          unsigned ss = s.u8();
          H.depth[c] = (int)(ss & 0x7F) + 1;
          H.is_signed[c] = (ss >> 7) & 1;
          H.sub_x[c] = (int)s.u8();
          H.sub_y[c] = (int)s.u8();
        }
        if (!s.ok) return PARSE_ERR_TRUNCATED;
        have_siz = true;
        break;
      }
      case 0xFF52:  // COD
        rc = read_cod(s, H, coc_set);
        have_cod = true;
        break;
      case 0xFF53:  // COC
        rc = read_coc(s, H, coc_set);
        break;
      case 0xFF5C:  // QCD
      case 0xFF5D:  // QCC
        rc = read_qcx(s, m == 0xFF5D, H, qcc_set);
        if (m == 0xFF5C) have_qcd = true;
        break;
      case 0xFF5E:  // RGN
        rc = read_rgn(s, H);
        break;
      case 0xFF5F:  // POC
        rc = read_poc(s, H.ncomp, H.poc);
        break;
      case 0xFF60:  // PPM: packed packet headers of every tile-part, in Zppm order
        if (s.left() < 1) return PARSE_ERR_TRUNCATED;
        ppm.push_back({(int)s.p[0], {s.p + 1, s.left() - 1}});
        break;
      default:  // COM, TLM, PLM, CRG and others are skipped
        break;
    }
    if (rc != PARSE_OK) return rc;
  }
  if (!have_siz || !have_cod || !have_qcd) return PARSE_ERR_MARKER;
  if (H.x0 < 0 || H.y0 < 0 || H.tx0 < 0 || H.ty0 < 0) return PARSE_ERR_INVALID;  // above 2^31
  if (H.width <= H.x0 || H.height <= H.y0 || H.tile_w <= 0 || H.tile_h <= 0) return PARSE_ERR_INVALID;
  // the tile grid starts at or above-left of the image origin and its first tile meets the
  // image (T.800 A.5.1)
  if (H.tx0 > H.x0 || H.ty0 > H.y0 || (int64_t)H.tx0 + H.tile_w <= H.x0 || (int64_t)H.ty0 + H.tile_h <= H.y0)
    return PARSE_ERR_INVALID;
  // tile indices are 16-bit, 65535 excluded (T.800 A.4.2)
  if ((int64_t)H.ntx() * H.nty() > 65535) return PARSE_ERR_INVALID;
  for (int c = 0; c < H.ncomp; ++c) {
    // component separation XRsiz / YRsiz (T.800 A.5.1: 1..255); sub-sampled components are
    // decoded on their own grids (B.2-B.3) and replicated onto the picture grid on output
    if (H.sub_x[c] < 1 || H.sub_y[c] < 1) return PARSE_ERR_INVALID;
    if (H.depth[c] > 16 || H.depth[c] != H.depth[0]) return PARSE_ERR_UNSUPPORTED;
    // signed samples take no DC level shift (T.800 G.1.2); the output stages apply the
    // unsigned shift, so such pictures are refused rather than decoded wrongly
    if (H.is_signed[c]) return PARSE_ERR_UNSUPPORTED;
  }
  int rc = finish_coding(H, nullptr);
  if (rc != PARSE_OK) return rc;
  if (!ppm.empty()) {
    std::stable_sort(ppm.begin(), ppm.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    for (auto &seg : ppm) H.ppm.insert(H.ppm.end(), seg.second.first, seg.second.first + seg.second.second);
    H.has_ppm = true;
  }
  H.header_len = (size_t)(r.p - data);
  return PARSE_OK;
}

namespace {
constexpr size_t kPoolMinBytes = size_t(1) << 20, kPoolMaxBytes = size_t(512) << 20;
constexpr size_t kPoolMaxBuffers = 8;
std::mutex g_pool_mu;
std::vector<ByteBuffer> g_pool;
size_t g_pool_bytes = 0;
}  // namespace

ByteBuffer take_plan_bytes(size_t capacity) {
  ByteBuffer v;
  if (capacity >= kPoolMinBytes) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    size_t best = g_pool.size();
    for (size_t i = 0; i < g_pool.size(); ++i)
      if (g_pool[i].capacity() >= capacity && (best == g_pool.size() || g_pool[i].capacity() < g_pool[best].capacity()))
        best = i;
    if (best < g_pool.size()) {
      v = std::move(g_pool[best]);
      g_pool.erase(g_pool.begin() + (std::ptrdiff_t)best);
      g_pool_bytes -= v.capacity();
      v.clear();
      return v;
    }
    capacity += capacity / 8;  // room for a slightly larger picture when it comes back
  }
  v.reserve(capacity);
  return v;
}

void give_plan_bytes(ByteBuffer &&bytes) {
  if (bytes.capacity() < kPoolMinBytes) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (g_pool.size() >= kPoolMaxBuffers || g_pool_bytes + bytes.capacity() > kPoolMaxBytes) return;
  g_pool_bytes += bytes.capacity();
  g_pool.push_back(std::move(bytes));
}

int build_plan(const uint8_t *data, size_t len, const DecodeOptions &opt, ImagePlan &P) {
  P = ImagePlan();
  P.bytes = take_plan_bytes(len);  // the coded bytes of every block are a subset of the codestream
  int st = parse_header(data, len, P.hdr);
  if (st != PARSE_OK) return st;
  const StreamHeader &H = P.hdr;
  const int ntx = H.ntx(), nty = H.nty(), ntiles = ntx * nty;

  // ---- gather tile-parts per tile (T.800 A.4): bodies, the tile's own coding parameters
  // (COD/COC/QCD/QCC/RGN of its first tile-part), its POC volumes and its packed packet
  // headers (PPT segments, or this tile-part's share of the main header's PPM data)
  std::vector<std::vector<std::pair<const uint8_t *, size_t>>> tparts(ntiles);
  std::vector<std::unique_ptr<StreamHeader>> thdr(ntiles);
  std::vector<std::vector<uint8_t>> packed(ntiles);
  std::vector<char> has_packed(ntiles, H.has_ppm ? 1 : 0);
  {
    Reader r{data + H.header_len, data + len};
    size_t ppm_pos = 0;
    std::vector<bool> tile_seen(ntiles, false), tile_poc(ntiles, false);
    for (;;) {
      if (r.left() < 2) return PARSE_ERR_TRUNCATED;
      unsigned m = r.u16();
      if (m == 0xFFD9) break;
      if (m != 0xFF90) return PARSE_ERR_MARKER;
      const uint8_t *sot = r.p - 2;
      unsigned lsot = r.u16();
      unsigned isot = r.u16();
      uint32_t psot = r.u32();
      r.u8();  // TPsot
      r.u8();  // TNsot
      if (!r.ok || lsot != 10) return PARSE_ERR_TRUNCATED;
      if ((int)isot >= ntiles) return PARSE_ERR_INVALID;
      const bool first = !tile_seen[isot];
      tile_seen[isot] = true;
      // precedence inside a tile: tile COC > tile COD > main COC > main COD (likewise QCC/QCD)
      bool tcoc[J2K_MAX_COMPONENTS] = {false}, tqcc[J2K_MAX_COMPONENTS] = {false};
      for (;;) {
        if (r.left() < 2) return PARSE_ERR_TRUNCATED;
        unsigned mm = r.u16();
        if (mm == 0xFF93) break;
        if (r.left() < 2) return PARSE_ERR_TRUNCATED;
        unsigned l = r.u16();
        if (l < 2 || l - 2 > r.left()) return PARSE_ERR_TRUNCATED;
        Reader s{r.p, r.p + (l - 2)};
        r.p += l - 2;
        int rc = PARSE_OK;
        const bool coding = mm == 0xFF52 || mm == 0xFF53 || mm == 0xFF5C || mm == 0xFF5D || mm == 0xFF5E;
        if (coding && !first) continue;  // only the first tile-part may carry them
        if ((coding || mm == 0xFF5F) && !thdr[isot]) {
          thdr[isot].reset(new StreamHeader(H));  // the main header's values, POC included
          thdr[isot]->ppm.clear();
        }
        StreamHeader *T = thdr[isot].get();
        switch (mm) {
          case 0xFF52: rc = read_cod(s, *T, tcoc); break;
          case 0xFF53: rc = read_coc(s, *T, tcoc); break;
          case 0xFF5C: rc = read_qcx(s, false, *T, tqcc); break;
          case 0xFF5D: rc = read_qcx(s, true, *T, tqcc); break;
          case 0xFF5E: rc = read_rgn(s, *T); break;
          case 0xFF5F:  // POC: the tile's volumes (from all its tile-parts) replace the main header's
            if (!tile_poc[isot]) T->poc.clear();
            tile_poc[isot] = true;
            rc = read_poc(s, H.ncomp, T->poc);
            break;
          case 0xFF61:  // PPT
            if (H.has_ppm) return PARSE_ERR_INVALID;
            if (s.left() < 1) return PARSE_ERR_TRUNCATED;
            packed[isot].insert(packed[isot].end(), s.p + 1, s.end);
            has_packed[isot] = 1;
            break;
          default:  // PLT, COM and others are skipped
            break;
        }
        if (rc != PARSE_OK) return rc;
      }
      if (H.has_ppm) {  // Nppm, then this tile-part's packet headers
        if (H.ppm.size() - ppm_pos < 4) return PARSE_ERR_INVALID;
        const uint8_t *q = H.ppm.data() + ppm_pos;
        const size_t n = ((size_t)q[0] << 24) | ((size_t)q[1] << 16) | ((size_t)q[2] << 8) | q[3];
        if (H.ppm.size() - ppm_pos - 4 < n) return PARSE_ERR_INVALID;
        packed[isot].insert(packed[isot].end(), q + 4, q + 4 + n);
        ppm_pos += 4 + n;
      }
      const uint8_t *body = r.p;
      const uint8_t *tend;
      if (psot == 0) {
        // to EOC
        tend = data + len;
        if (len >= 2 && data[len - 2] == 0xFF && data[len - 1] == 0xD9) tend -= 2;
      } else if ((size_t)(data + len - sot) < psot) {
        tend = data + len;  // truncated stream: keep the bytes that are there
        psot = 0;
      } else {
        tend = sot + psot;
      }
      if (tend < body) return PARSE_ERR_INVALID;
      tparts[isot].push_back({body, (size_t)(tend - body)});
      r.p = tend;
      if (psot == 0) break;
    }
  }
  for (int t = 0; t < ntiles; ++t)
    if (thdr[t]) {
      const int rc = finish_coding(*thdr[t], &H);
      if (rc != PARSE_OK) return rc;
    }
  auto tile_header = [&](int t) -> const StreamHeader & { return thdr[t] ? *thdr[t] : H; };

  int discard = opt.discard_levels;
  for (int t = 0; t < ntiles; ++t)
    for (int c = 0; c < H.ncomp; ++c) discard = std::min(discard, tile_header(t).levels[c]);
  if (discard < 0) discard = 0;
  P.discard = discard;

  // ---- geometry and Tier-2 per tile.  Tiles are independent: each fills a TileOut with
  // tile-relative offsets, on `opt.threads` host threads; the outputs are then merged in
  // tile order, so the plan does not depend on the thread count.
  struct TileOut {
    std::vector<j2k_tilecomp> tcs;
    std::vector<j2k_cblk> cblks;
    std::vector<uint32_t> seglens;
    std::vector<std::pair<const uint8_t *, uint32_t>> spans;  // coded bytes, block after block
    uint64_t coef = 0;
    size_t bytes = 0;
  };
  std::vector<TileOut> outs(ntiles);
  P.out_w = H.out_w(discard);
  P.out_h = H.out_h(discard);
  auto process_tile = [&](int t, TileOut &out) -> int {
    uint64_t coef_total = 0;
    const StreamHeader &TH = tile_header(t);
    const int maxlayers = opt.max_layers > 0 ? std::min(opt.max_layers, TH.layers) : TH.layers;
    int tx = t % ntx, ty = t / ntx;
    const int tx0 = (int)std::max<int64_t>(TH.tx0 + (int64_t)tx * TH.tile_w, TH.x0);
    const int ty0 = (int)std::max<int64_t>(TH.ty0 + (int64_t)ty * TH.tile_h, TH.y0);
    const int tx1 = (int)std::min<int64_t>(TH.tx0 + (int64_t)(tx + 1) * TH.tile_w, TH.width);
    const int ty1 = (int)std::min<int64_t>(TH.ty0 + (int64_t)(ty + 1) * TH.tile_h, TH.height);
    std::vector<TCState> tcs(TH.ncomp);
    size_t tile_blocks = 0;
    for (int c = 0; c < TH.ncomp; ++c) {
      TCState &TC = tcs[c];
      TC.comp = c;
      // the tile on component c's own grid (T.800 B.3: ceil of the reference-grid bounds
      // over XRsiz / YRsiz)
      TC.x0 = ceil_div(tx0, TH.sub_x[c]);
      TC.y0 = ceil_div(ty0, TH.sub_y[c]);
      TC.x1 = ceil_div(tx1, TH.sub_x[c]);
      TC.y1 = ceil_div(ty1, TH.sub_y[c]);
      TC.levels = TH.levels[c];
      const int L = TC.levels;
      TC.res.resize(L + 1);
      for (int r = 0; r <= L; ++r) {
        ResState &R = TC.res[r];
        int nb = L - r;
        R.x0 = ceil_div_pow2(TC.x0, nb);
        R.y0 = ceil_div_pow2(TC.y0, nb);
        R.x1 = ceil_div_pow2(TC.x1, nb);
        R.y1 = ceil_div_pow2(TC.y1, nb);
        // the device DWT synthesises every resolution r >= 1 with its first sample low-pass,
        // i.e. from an even origin (the reference's HDWT ignores xParity as well,
        // bmi_cpu_dwt_decoder.cpp:2609); the coarsest LL band (r = 0) is never synthesised
        if (r > 0 && ((R.x0 & 1) || (R.y0 & 1))) return PARSE_ERR_UNSUPPORTED;
        int ppx = TH.ppx[c][r], ppy = TH.ppy[c][r];
        if (R.x1 > R.x0 && R.y1 > R.y0) {
          R.npx = ((R.x1 + (1 << ppx) - 1) >> ppx) - (R.x0 >> ppx);
          R.npy = ((R.y1 + (1 << ppy) - 1) >> ppy) - (R.y0 >> ppy);
        }
        int nbands = r == 0 ? 1 : 3;
        R.bands.resize(nbands);
        int cbw = r == 0 ? std::min(TH.cbw_exp[c], ppx) : std::min(TH.cbw_exp[c], ppx - 1);
        int cbh = r == 0 ? std::min(TH.cbh_exp[c], ppy) : std::min(TH.cbh_exp[c], ppy - 1);
        for (int b = 0; b < nbands; ++b) {
          BandState &B = R.bands[b];
          B.type = r == 0 ? 0 : b + 1;
          int lev = r == 0 ? L : L - r + 1;
          int xob = B.type & 1, yob = (B.type >> 1) & 1;
          int sh = lev > 0 ? 1 << (lev - 1) : 0;
          B.x0 = ceil_div_pow2(TC.x0 - sh * xob, lev);
          B.y0 = ceil_div_pow2(TC.y0 - sh * yob, lev);
          B.x1 = ceil_div_pow2(TC.x1 - sh * xob, lev);
          B.y1 = ceil_div_pow2(TC.y1 - sh * yob, lev);
          B.cbw_exp = cbw;
          B.cbh_exp = cbh;
          int bi = r == 0 ? 0 : 1 + 3 * (r - 1) + b;
          B.spqcd = TH.steps[c][bi];
          int G = TH.guard[c];
          if (TH.reversible[c]) {
            B.mb = (int)B.spqcd + G - 1;
            B.gain = 0.f;
          } else {
            B.mb = std::max(0, (int)(B.spqcd >> 11) + G - 1);
            B.gain = irrev_band_gain(B.spqcd, TH.depth[c], B.type, L == 0);
          }
          // position in the Mallat region of the tile-component
          if (r == 0) {
            B.off_x = B.off_y = 0;
          } else {
            const ResState &Rl = TC.res[r - 1];
            B.off_x = xob ? (Rl.x1 - Rl.x0) : 0;
            B.off_y = yob ? (Rl.y1 - Rl.y0) : 0;
          }
          // precincts and code-blocks
          int np = R.npx * R.npy;
          B.prec_cbs.assign(np, {});
          B.incl.assign(np, TagTree());
          B.zbp.assign(np, TagTree());
          if (B.x1 <= B.x0 || B.y1 <= B.y0) continue;
          // every code-block lies in one precinct (precinct edges are on the block grid)
          B.cbs.reserve((size_t)(((B.x1 + (1 << cbw) - 1) >> cbw) - (B.x0 >> cbw)) *
                        (size_t)(((B.y1 + (1 << cbh) - 1) >> cbh) - (B.y0 >> cbh)));
          // precinct size in band coordinates
          int pbx = r == 0 ? ppx : ppx - 1, pby = r == 0 ? ppy : ppy - 1;
          int px0 = R.x0 >> ppx, py0 = R.y0 >> ppy;
          for (int pj = 0; pj < R.npy; ++pj)
            for (int pi = 0; pi < R.npx; ++pi) {
              int p = pj * R.npx + pi;
              // precinct extent in band coordinates
              int bx0 = std::max(B.x0, (px0 + pi) << pbx), bx1 = std::min(B.x1, (px0 + pi + 1) << pbx);
              int by0 = std::max(B.y0, (py0 + pj) << pby), by1 = std::min(B.y1, (py0 + pj + 1) << pby);
              if (bx1 <= bx0 || by1 <= by0) continue;
              int cx0 = bx0 >> cbw, cx1 = (bx1 + (1 << cbw) - 1) >> cbw;
              int cy0 = by0 >> cbh, cy1 = (by1 + (1 << cbh) - 1) >> cbh;
              B.incl[p].build(cx1 - cx0, cy1 - cy0);
              B.zbp[p].build(cx1 - cx0, cy1 - cy0);
              B.prec_cbs[p].reserve((size_t)(cx1 - cx0) * (cy1 - cy0));
              for (int cy = cy0; cy < cy1; ++cy)
                for (int cx = cx0; cx < cx1; ++cx) {
                  CbState cb;
                  int gx0 = std::max(bx0, cx << cbw), gx1 = std::min(bx1, (cx + 1) << cbw);
                  int gy0 = std::max(by0, cy << cbh), gy1 = std::min(by1, (cy + 1) << cbh);
                  cb.x0 = gx0 - B.x0;
                  cb.y0 = gy0 - B.y0;
                  cb.w = gx1 - gx0;
                  cb.h = gy1 - gy0;
                  B.prec_cbs[p].push_back((int)B.cbs.size());
                  B.cbs.push_back(cb);
                  ++tile_blocks;
                }
            }
        }
      }
    }

    // ---- packets
    std::vector<Piece> pieces;  // the tile's coded pieces, linked per block
    std::vector<SegLen> segs;   // the tile's codeword-segment lengths, linked per block
    pieces.reserve(tile_blocks * (size_t)std::min(TH.layers, 8));
    segs.reserve(tile_blocks * (size_t)std::min(TH.layers, 8));
    const uint8_t *cur = nullptr, *end = nullptr;
    size_t part = 0;
    auto next_part = [&]() -> bool {
      while (part < tparts[t].size()) {
        cur = tparts[t][part].first;
        end = cur + tparts[t][part].second;
        ++part;
        if (cur < end) return true;
      }
      cur = end = nullptr;
      return false;
    };
    next_part();
    bool stream_end = false;
    // one packet's code-block contributions; reused across packets (no allocation per
    // contribution): segment lengths live in one flat buffer
    struct Contrib {
      CbState *cb;
      uint32_t lens_at, nlens;
      int newpasses;
      int first_seg_new;  // whether the first piece opens a new segment
    };
    std::vector<Contrib> contribs;
    std::vector<uint32_t> lens;
    // packet headers: in the tile data, or packed (PPM / PPT) in a stream of their own
    const bool pk = has_packed[t] != 0;
    const uint8_t *hcur = pk ? packed[t].data() : nullptr;
    const uint8_t *const hend = pk ? packed[t].data() + packed[t].size() : nullptr;
    // reads the packet of layer l, resolution r, component c, precinct p (which exist)
    auto read_packet = [&](int l, int r, int c, int p) -> int {
      TCState &TC = tcs[c];
      ResState &R = TC.res[r];
      if (stream_end) return PARSE_OK;
      while (cur && cur >= end) next_part();
      if (pk ? hcur >= hend : !cur) {
        stream_end = true;  // truncated tile: remaining packets are empty
        return PARSE_OK;
      }
      if (TH.sop && cur && end - cur >= 6 && cur[0] == 0xFF && cur[1] == 0x91) cur += 6;
      BitReader br = pk ? BitReader{hcur, hend} : BitReader{cur, end};
      contribs.clear();
      lens.clear();
      const int style = TH.cbstyle[c];
      const bool one_segment = !(style & (J2K_CB_BYPASS | J2K_CB_TERMALL));
      if (br.bit()) {
        for (auto &B : R.bands) {
          if (B.prec_cbs.empty() || B.prec_cbs[p].empty()) continue;
          const std::vector<int> &members = B.prec_cbs[p];
          TagTree &incl_tree = B.incl[p];
          TagTree &zbp_tree = B.zbp[p];
          for (size_t k = 0; k < members.size(); ++k) {
            CbState &cb = B.cbs[members[k]];
            int incl;
            if (!cb.included) incl = incl_tree.decode(br, (int)k, l + 1);
            else incl = br.bit();
            if (br.overrun) return PARSE_ERR_PACKET;
            if (!incl) continue;
            if (!cb.included) {
              int i = 0;
              while (!zbp_tree.decode(br, (int)k, i)) {
                ++i;
                if (br.overrun || i > 74) return PARSE_ERR_PACKET;
              }
              cb.missing = i - 1;
              cb.included = true;
            }
            int n;
            if (!br.bit()) n = 1;
            else if (!br.bit()) n = 2;
            else {
              n = (int)br.bits(2);
              if (n < 3) n += 3;
              else {
                n = (int)br.bits(5);
                if (n < 31) n += 6;
                else n = 37 + (int)br.bits(7);
              }
            }
            while (br.bit()) {
              if (++cb.lblock > 32 || br.overrun) return PARSE_ERR_PACKET;
            }
            Contrib ct{&cb, (uint32_t)lens.size(), 0, n, 0};
            if (one_segment) {  // every pass in the block's single codeword segment
              const int nb = cb.lblock + floor_log2((uint32_t)n);
              if (nb > 32) return PARSE_ERR_PACKET;
              lens.push_back(br.bits(nb));
              ct.first_seg_new = cb.passes == 0;
            } else {
              int s = cb.passes;
              while (s < cb.passes + n) {
                const int e = std::min(next_seg_start(style, s), cb.passes + n);
                const int nb = cb.lblock + floor_log2((uint32_t)(e - s));
                if (nb > 32) return PARSE_ERR_PACKET;
                lens.push_back(br.bits(nb));
                if (s == cb.passes) ct.first_seg_new = seg_starts(style, s);
                s = e;
              }
            }
            if (br.overrun) return PARSE_ERR_PACKET;
            ct.nlens = (uint32_t)lens.size() - ct.lens_at;
            contribs.push_back(ct);
          }
        }
      }
      br.align();
      const uint8_t *&hp = pk ? hcur : cur;
      const uint8_t *const he = pk ? hend : end;
      hp = br.p;
      if (TH.eph && he - hp >= 2 && hp[0] == 0xFF && hp[1] == 0x92) hp += 2;
      const bool keep = l < maxlayers;
      for (auto &ct : contribs) {
        CbState &cb = *ct.cb;
        for (uint32_t i = 0; i < ct.nlens; ++i) {
          uint32_t L = lens[ct.lens_at + i];
          if ((size_t)(end - cur) < L) {
            // truncated packet body: keep what is there, stop the tile
            L = (uint32_t)(end - cur);
            stream_end = true;
          }
          if (keep) {
            if (L) {
              const int32_t at = (int32_t)pieces.size();
              pieces.push_back({cur, L, -1});
              if (cb.piece_tail >= 0) pieces[cb.piece_tail].next = at;
              else cb.piece_head = at;
              cb.piece_tail = at;
            }
            const bool newseg = (i > 0) || ct.first_seg_new;
            if (newseg || cb.nseg == 0) {
              const int32_t at = (int32_t)segs.size();
              segs.push_back({L, -1});
              if (cb.seg_tail >= 0) segs[cb.seg_tail].next = at;
              else cb.seg_head = at;
              cb.seg_tail = at;
              cb.nseg++;
            } else {
              segs[cb.seg_tail].len += L;
            }
          }
          cur += L;
        }
        cb.passes += ct.newpasses;
        if (keep) cb.kept = cb.passes;
        if (cb.passes > 255) return PARSE_ERR_PACKET;
      }
      return PARSE_OK;
    };

    // ---- packet order (T.800 B.12): the tile's POC volumes, else the main header's, else
    // the COD progression over everything.  Each packet is read once: a volume skips the
    // layers of a precinct that an earlier volume has read.
    int maxL = 0;
    for (int c = 0; c < TH.ncomp; ++c) maxL = std::max(maxL, tcs[c].levels);
    std::vector<std::vector<std::vector<int>>> next_layer(TH.ncomp);
    for (int c = 0; c < TH.ncomp; ++c) {
      next_layer[c].resize(tcs[c].levels + 1);
      for (int r = 0; r <= tcs[c].levels; ++r) next_layer[c][r].assign(tcs[c].res[r].npx * tcs[c].res[r].npy, 0);
    }
    auto nprec = [&](int r, int c) -> int { return r <= tcs[c].levels ? (int)next_layer[c][r].size() : 0; };
    auto visit = [&](int l, int r, int c, int p) -> int {
      int &nl = next_layer[c][r][p];
      if (l < nl) return PARSE_OK;
      nl = l + 1;
      return read_packet(l, r, c, p);
    };
    // position-driven orders visit each precinct at the reference-grid point of its
    // upper-left corner inside the tile (T.800 B.12.1.3-B.12.1.5)
    struct PrecinctVisit {
      int64_t y, x;
      int r, c, p;
    };
    std::vector<PrecinctVisit> pv;
    std::vector<PocEntry> vols = TH.poc;
    if (vols.empty()) vols.push_back({0, 0, TH.layers, maxL + 1, TH.ncomp, TH.progression});
    int rc = PARSE_OK;
    // a tile whose data (or packed headers) ran out has no packet left to read
    auto go = [&]() { return rc == PARSE_OK && !stream_end; };
    for (const PocEntry &v : vols) {
      const int lye = std::min(v.lye, TH.layers), re = std::min(v.re, maxL + 1), ce = std::min(v.ce, TH.ncomp);
      const int rs = v.rs, cs = v.cs;
      if (rs >= re || cs >= ce || lye <= 0) continue;
      if (v.prog == 0) {  // LRCP
        for (int l = 0; l < lye && go(); ++l)
          for (int r = rs; r < re && go(); ++r)
            for (int c = cs; c < ce && go(); ++c)
              for (int p = 0; p < nprec(r, c) && go(); ++p) rc = visit(l, r, c, p);
      } else if (v.prog == 1) {  // RLCP
        for (int r = rs; r < re && go(); ++r)
          for (int l = 0; l < lye && go(); ++l)
            for (int c = cs; c < ce && go(); ++c)
              for (int p = 0; p < nprec(r, c) && go(); ++p) rc = visit(l, r, c, p);
      } else {  // RPCL, PCRL, CPRL
        pv.clear();
        for (int c = cs; c < ce; ++c) {
          const TCState &TC = tcs[c];
          for (int r = rs; r < re && r <= TC.levels; ++r) {
            const ResState &R = TC.res[r];
            if (R.npx * R.npy == 0) continue;
            const int lv = TC.levels - r, ppx = TH.ppx[c][r], ppy = TH.ppy[c][r];
            const int64_t rx0 = (int64_t)R.x0 << lv, ry0 = (int64_t)R.y0 << lv;
            const int64_t spx = (int64_t)1 << (ppx + lv), spy = (int64_t)1 << (ppy + lv);
            const int px0 = R.x0 >> ppx, py0 = R.y0 >> ppy;
            // reference-grid coordinates: component units times XRsiz / YRsiz; a precinct
            // starting before the tile is visited at the tile's own corner
            const int64_t dx = TH.sub_x[c], dy = TH.sub_y[c];
            for (int pj = 0; pj < R.npy; ++pj) {
              const int64_t y = pj ? (int64_t)(py0 + pj) * spy * dy : ((ry0 % spy) ? ty0 : ry0 * dy);
              for (int pi = 0; pi < R.npx; ++pi) {
                const int64_t x = pi ? (int64_t)(px0 + pi) * spx * dx : ((rx0 % spx) ? tx0 : rx0 * dx);
                pv.push_back({y, x, r, c, pj * R.npx + pi});
              }
            }
          }
        }
        const int prog = v.prog;
        std::sort(pv.begin(), pv.end(), [prog](const PrecinctVisit &a, const PrecinctVisit &b) {
          if (prog == 2) {  // RPCL: resolution, y, x, component
            if (a.r != b.r) return a.r < b.r;
            if (a.y != b.y) return a.y < b.y;
            if (a.x != b.x) return a.x < b.x;
            return a.c < b.c;
          }
          if (prog == 4 && a.c != b.c) return a.c < b.c;  // CPRL: component first
          if (a.y != b.y) return a.y < b.y;
          if (a.x != b.x) return a.x < b.x;
          if (prog == 3 && a.c != b.c) return a.c < b.c;  // PCRL: y, x, component, resolution
          return a.r < b.r;
        });
        for (const PrecinctVisit &q : pv)
          for (int l = 0; l < lye && go(); ++l) rc = visit(l, q.r, q.c, q.p);
      }
      if (!go()) break;
    }
    if (rc != PARSE_OK) return rc;

    // ---- emit plan entries for this tile (offsets relative to the tile)
    size_t tile_bytes = 0;
    out.spans.reserve(pieces.size());
    out.cblks.reserve(tile_blocks);
    out.seglens.reserve(segs.size());
    for (int c = 0; c < TH.ncomp; ++c) {
      TCState &TC = tcs[c];
      if ((opt.ignore_components >> c) & 1) continue;
      const int L = TC.levels;
      const int keep = L - discard;  // resolutions 0..keep are reconstructed
      j2k_tilecomp tc{};
      tc.comp = c;
      tc.tile = t;
      tc.levels = keep;
      const ResState &Rtop = TC.res[keep];
      // relative to the component's own image origin at the output resolution
      tc.x0 = Rtop.x0 - ceil_div_pow2(ceil_div(TH.x0, TH.sub_x[c]), discard);
      tc.y0 = Rtop.y0 - ceil_div_pow2(ceil_div(TH.y0, TH.sub_y[c]), discard);
      tc.w = Rtop.x1 - Rtop.x0;
      tc.h = Rtop.y1 - Rtop.y0;
      for (int r = 0; r <= keep; ++r) {
        tc.res_w[r] = TC.res[r].x1 - TC.res[r].x0;
        tc.res_h[r] = TC.res[r].y1 - TC.res[r].y0;
      }
      tc.coef_off = coef_total;
      coef_total += (uint64_t)tc.w * tc.h;
      out.tcs.push_back(tc);
      for (int r = 0; r <= keep; ++r) {
        for (auto &B : TC.res[r].bands) {
          for (auto &cb : B.cbs) {
            j2k_cblk d{};
            d.w = (uint16_t)cb.w;
            d.h = (uint16_t)cb.h;
            d.band = (uint8_t)B.type;
            d.spqcd = B.spqcd;
            d.mb = (uint8_t)std::min(B.mb, 255);
            d.missing = (uint8_t)std::min(cb.missing, 255);
            d.num_passes = (uint8_t)cb.kept;
            d.flags = (uint8_t)((TH.cbstyle[c] & 0x3F) | (TH.reversible[c] ? 0 : J2K_CB_IRREV));
            d.gain = B.gain;
            d.out_stride = (uint32_t)tc.w;
            d.out_off = tc.coef_off + (uint64_t)(B.off_y + cb.y0) * tc.w + (B.off_x + cb.x0);
            d.data_off = (uint32_t)tile_bytes;
            uint32_t total = 0;
            for (int32_t i = cb.piece_head; i >= 0; i = pieces[i].next) {
              total += pieces[i].len;
              out.spans.push_back({pieces[i].p, pieces[i].len});
            }
            tile_bytes += total;
            d.data_len = total;
            d.seg_off = (uint32_t)out.seglens.size();
            d.nseg = (uint8_t)std::min<uint32_t>(cb.nseg, 255);
            for (int32_t i = cb.seg_head; i >= 0; i = segs[i].next) out.seglens.push_back(segs[i].len);
            if (cb.kept == 0) d.nseg = 0;
            out.cblks.push_back(d);
          }
        }
      }
    }
    out.coef = coef_total;
    out.bytes = tile_bytes;
    return PARSE_OK;
  };

  // run the tiles; the error of the first failing tile in tile order is reported
  std::vector<int> tile_rc(ntiles, PARSE_OK);
  const int nthreads = std::max(1, std::min(opt.threads, ntiles));
  if (nthreads <= 1) {
    for (int t = 0; t < ntiles; ++t)
      if ((tile_rc[t] = process_tile(t, outs[t])) != PARSE_OK) return tile_rc[t];
  } else {
    std::atomic<int> next{0};
    std::mutex ex_mu;
    std::exception_ptr ex;
    auto worker = [&]() {
      for (int t; (t = next.fetch_add(1)) < ntiles;) {
        try {
          tile_rc[t] = process_tile(t, outs[t]);
        } catch (...) {  // rethrown on the calling thread
          std::lock_guard<std::mutex> lk(ex_mu);
          if (!ex) ex = std::current_exception();
          tile_rc[t] = PARSE_ERR_INVALID;
        }
      }
    };
    std::vector<std::thread> th;
    for (int i = 1; i < nthreads; ++i) {
      try {
        th.emplace_back(worker);
      } catch (...) {
        break;
      }
    }
    worker();
    for (auto &x : th) x.join();
    if (ex) std::rethrow_exception(ex);
    for (int t = 0; t < ntiles; ++t)
      if (tile_rc[t] != PARSE_OK) return tile_rc[t];
  }

  // ---- merge in tile order
  size_t n_tcs = 0, n_cblks = 0, n_segs = 0, n_bytes = 0;
  for (const TileOut &o : outs) {
    n_tcs += o.tcs.size();
    n_cblks += o.cblks.size();
    n_segs += o.seglens.size();
    n_bytes += o.bytes;
  }
  if (n_bytes > 0xFFFFFFF0ull || n_segs > 0xFFFFFFF0ull) return PARSE_ERR_UNSUPPORTED;
  P.tilecomps.reserve(n_tcs);
  P.cblks.reserve(n_cblks);
  P.seglens.reserve(n_segs);
  P.bytes.resize(n_bytes);
  uint64_t coef_total = 0;
  size_t byte_base = 0;
  std::vector<CopyChunk> chunks;
  for (TileOut &o : outs) {
    const uint32_t seg_base = (uint32_t)P.seglens.size();
    if (ntiles == 1) {  // one tile: every offset is already the plan's
      P.tilecomps = std::move(o.tcs);
      P.cblks = std::move(o.cblks);
      P.seglens = std::move(o.seglens);
    } else {
      for (j2k_tilecomp tc : o.tcs) {
        tc.coef_off += coef_total;
        P.tilecomps.push_back(tc);
      }
      for (j2k_cblk d : o.cblks) {
        d.out_off += coef_total;
        d.data_off += (uint32_t)byte_base;
        d.seg_off += seg_base;
        P.cblks.push_back(d);
      }
      P.seglens.insert(P.seglens.end(), o.seglens.begin(), o.seglens.end());
    }
    // chunks of about 1 MB of this tile's spans
    uint8_t *dst = P.bytes.data() + byte_base;
    const auto *b = o.spans.data(), *e = o.spans.data() + o.spans.size();
    while (b != e) {
      const auto *k = b;
      size_t n = 0;
      while (k != e && n < (size_t(1) << 20)) n += (k++)->second;
      chunks.push_back({dst, b, k});
      dst += n;
      b = k;
    }
    coef_total += o.coef;
    byte_base += o.bytes;
  }
  copy_chunks(chunks, n_bytes);

  j2k_image_info &I = P.info;
  I.width = P.out_w;
  I.height = P.out_h;
  I.ncomp = H.ncomp;
  I.bitdepth = H.depth[0];
  I.is_signed = H.is_signed[0];
  I.tile_w = H.tile_w;
  I.tile_h = H.tile_h;
  I.ntiles_x = ntx;
  I.ntiles_y = nty;
  I.levels = H.levels[0] - discard;
  I.reversible = H.reversible[0];
  I.mct = H.mct;
  I.layers = H.layers;
  I.progression = H.progression;
  I.cbw = 1 << H.cbw_exp[0];
  I.cbh = 1 << H.cbh_exp[0];
  I.cbstyle = H.cbstyle[0];
  I.guard_bits = H.guard[0];
  I.num_cblks = (int32_t)P.cblks.size();
  I.num_tilecomps = (int32_t)P.tilecomps.size();
  I.num_segs = (int32_t)P.seglens.size();
  I.coded_bytes = P.bytes.size();
  I.coef_elems = coef_total;
  I.origin_x = ceil_div_pow2(H.x0, discard);
  I.origin_y = ceil_div_pow2(H.y0, discard);
  for (int c = 0; c < H.ncomp; ++c) {
    I.sub_x[c] = H.sub_x[c];
    I.sub_y[c] = H.sub_y[c];
    const int cx0 = ceil_div(H.x0, H.sub_x[c]), cy0 = ceil_div(H.y0, H.sub_y[c]);
    I.comp_x0[c] = ceil_div_pow2(cx0, discard);
    I.comp_y0[c] = ceil_div_pow2(cy0, discard);
    I.comp_w[c] = ceil_div_pow2(ceil_div(H.width, H.sub_x[c]), discard) - I.comp_x0[c];
    I.comp_h[c] = ceil_div_pow2(ceil_div(H.height, H.sub_y[c]), discard) - I.comp_y0[c];
  }
  return PARSE_OK;
}

}  // namespace j2k
