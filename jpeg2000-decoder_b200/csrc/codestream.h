/*
 * codestream.h — host-side JPEG 2000 Part-1 front end: marker segments, tiles and
 * Tier-2 packet headers, producing a decode plan (plan.h) for the device.
 *
 * Mirrors the role of the reference's codestream layer, which stays on the host there too:
 * dec_syntax.cpp (SIZ/COD/COC/QCD/QCC/RGN/COM/POC/PPM parsing, :134-421; tile-part headers
 * with COD/COC/QCD/QCC/RGN/POC/PPT, :560-720), dec_packet.cpp (packet headers, pass
 * counts, Lblock, lengths, :66-221; progression orders :384-830),
 * dec_tagtree.cpp (tag trees), dec_init.cpp (tile / subband / code-block geometry,
 * :645-1056) and dec_jp2.cpp (JP2 wrapper, BMI_dec_info sizes, :420-597).
 */
#ifndef J2K_CODESTREAM_H
#define J2K_CODESTREAM_H

#include <cstddef>
#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "plan.h"

namespace j2k {

enum ParseStatus {
  PARSE_OK = 0,
  PARSE_ERR_TRUNCATED = -1,
  PARSE_ERR_MARKER = -2,
  PARSE_ERR_UNSUPPORTED = -3,
  PARSE_ERR_INVALID = -4,
  PARSE_ERR_PACKET = -5
};

struct DecodeOptions {
  int discard_levels = 0;    /* decode at 1/2^n resolution (reference mDwtDecodeTopLevel) */
  int max_layers = 0;        /* 0: all layers */
  unsigned ignore_components = 0; /* bit c set: component c is not decoded */
  int threads = 1;           /* host threads for the Tier-2 of a multi-tile picture */
};

/* std::allocator whose value-initialisation leaves the element unset: a plan's byte buffer
 * is resized and then filled by the Tier-2 copy, so zeroing it first is wasted work. */
template <class T>
struct NoInitAllocator : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAllocator<U>;
  };
  NoInitAllocator() = default;
  template <class U>
  NoInitAllocator(const NoInitAllocator<U> &) noexcept {}
  template <class U>
  void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new ((void *)p) U;
  }
  template <class U, class... A>
  void construct(U *p, A &&...a) {
    ::new ((void *)p) U(std::forward<A>(a)...);
  }
};
using ByteBuffer = std::vector<uint8_t, NoInitAllocator<uint8_t>>;

/* One progression volume of a POC marker (T.800 A.6.6): layers [0, lye), resolutions
 * [rs, re), components [cs, ce) in progression order `prog`. */
struct PocEntry {
  int rs, cs, lye, re, ce, prog;
};

/* Coding parameters of the main header, or of one tile (the main header's values with the
 * tile's own COD / COC / QCD / QCC / POC applied). */
struct StreamHeader {
  int width = 0, height = 0, x0 = 0, y0 = 0;
  int tile_w = 0, tile_h = 0, tx0 = 0, ty0 = 0;
  int ncomp = 0;
  int depth[J2K_MAX_COMPONENTS] = {0};
  int is_signed[J2K_MAX_COMPONENTS] = {0};
  int sub_x[J2K_MAX_COMPONENTS] = {0}, sub_y[J2K_MAX_COMPONENTS] = {0};
  int progression = 0, layers = 0, mct = 0;
  int levels[J2K_MAX_COMPONENTS] = {0};
  int cbw_exp[J2K_MAX_COMPONENTS] = {0}, cbh_exp[J2K_MAX_COMPONENTS] = {0};
  int cbstyle[J2K_MAX_COMPONENTS] = {0};
  int reversible[J2K_MAX_COMPONENTS] = {0};
  int ppx[J2K_MAX_COMPONENTS][J2K_MAX_LEVELS + 1] = {{0}}, ppy[J2K_MAX_COMPONENTS][J2K_MAX_LEVELS + 1] = {{0}};
  int sop = 0, eph = 0;
  int qstyle[J2K_MAX_COMPONENTS] = {0};
  int guard[J2K_MAX_COMPONENTS] = {0};
  uint16_t steps[J2K_MAX_COMPONENTS][3 * J2K_MAX_LEVELS + 1] = {{0}};  /* raw SPqcd/SPqcc values */
  int roi_shift[J2K_MAX_COMPONENTS] = {0};
  std::vector<PocEntry> poc;  /* progression volumes (empty: the COD order over everything) */
  std::vector<uint8_t> ppm;   /* main header only: PPM payloads (Nppm + packed headers per tile-part) */
  bool has_ppm = false;
  int jp2_colr_method = 0;  /* JP2 colour specification box: method (0 = none / raw codestream) */
  int jp2_colr_enum = 0;    /* its enumerated colour space (16 sRGB, 17 greyscale, 18 sYCC) */
  size_t header_len = 0;    /* bytes up to the first SOT */
  size_t cs_offset = 0;     /* offset of SOC inside the input (JP2 wrapper) */
  /* picture size: the reference grid from the image origin (x0, y0) to (width, height) */
  int image_w() const { return width - x0; }
  int image_h() const { return height - y0; }
  /* component c's grid at 1/2^d resolution (T.800 B.2): origin and size */
  int comp_x0(int c, int d) const { return (int)(((((int64_t)x0 + sub_x[c] - 1) / sub_x[c]) + (1LL << d) - 1) >> d); }
  int comp_y0(int c, int d) const { return (int)(((((int64_t)y0 + sub_y[c] - 1) / sub_y[c]) + (1LL << d) - 1) >> d); }
  int comp_w(int c, int d) const {
    return (int)(((((int64_t)width + sub_x[c] - 1) / sub_x[c]) + (1LL << d) - 1) >> d) - comp_x0(c, d);
  }
  int comp_h(int c, int d) const {
    return (int)(((((int64_t)height + sub_y[c] - 1) / sub_y[c]) + (1LL << d) - 1) >> d) - comp_y0(c, d);
  }
  /* picture size at 1/2^d resolution (T.800 B.5: ceil(width / 2^d) - ceil(x0 / 2^d)) */
  int out_w(int d) const { return (int)((((int64_t)width + (1LL << d) - 1) >> d) - (((int64_t)x0 + (1LL << d) - 1) >> d)); }
  int out_h(int d) const { return (int)((((int64_t)height + (1LL << d) - 1) >> d) - (((int64_t)y0 + (1LL << d) - 1) >> d)); }
  int ntx() const { return (int)(((int64_t)width - tx0 + tile_w - 1) / tile_w); }
  int nty() const { return (int)(((int64_t)height - ty0 + tile_h - 1) / tile_h); }
};

/* The full host-side plan of one image. */
struct ImagePlan {
  StreamHeader hdr;
  j2k_image_info info{};
  std::vector<j2k_cblk> cblks;
  std::vector<uint32_t> seglens;
  ByteBuffer bytes;                   /* Tier-1 bytes, block after block */
  std::vector<j2k_tilecomp> tilecomps;
  int out_w = 0, out_h = 0;           /* output size after discard_levels */
  int discard = 0;
};

int parse_header(const uint8_t *data, size_t len, StreamHeader &hdr);
/* Plan byte buffers of large pictures are recycled between plans (the coded bytes of a 4K
 * lossless picture fill tens of MB; a fresh buffer that size costs a page fault per 4 KB on
 * its first write, about a quarter of the Tier-2 time).  take_plan_bytes returns an empty
 * buffer with at least `capacity` bytes reserved; give_plan_bytes hands a plan's buffer back
 * (kept while the pool holds fewer than 8 buffers and under 512 MB). */
ByteBuffer take_plan_bytes(size_t capacity);
void give_plan_bytes(ByteBuffer &&bytes);
int build_plan(const uint8_t *data, size_t len, const DecodeOptions &opt, ImagePlan &plan);
const char *status_string(int status);

/* 9/7 band gain of the reference's gain folding, computed with the same float operations. */
float irrev_band_gain(uint16_t spqcd, int bitdepth, int band, int no_dwt);
/* Constant applied to the reconstructed LL of a coarser level before the next 9/7 level. */
float irrev_ll_gain();

}  // namespace j2k

/* opaque handle of the C ABI (include/j2k_gpu.h) */
struct j2k_plan {
  j2k::ImagePlan p;
};

#endif
