/*
 * plan_api.cpp — C ABI over the host front end (j2k_plan_* in include/j2k_gpu.h).
 * Host-only: it owns the Tier-2 result; the device code only ever sees the flat arrays.
 */
#include <new>
#include <utility>

#include "../../include/j2k_gpu.h"
#include "codestream.h"

extern "C" int j2k_plan_create_mt(const uint8_t *cs, size_t len, int discard_levels, int max_layers,
                                  unsigned ignore_components, int threads, j2k_plan **out) {
  if (!cs || !out || len < 2) return J2K_ERR_ARG;
  *out = nullptr;
  j2k_plan *p = new (std::nothrow) j2k_plan;
  if (!p) return J2K_ERR_NOMEM;
  j2k::DecodeOptions opt;
  opt.discard_levels = discard_levels < 0 ? 0 : discard_levels;
  opt.max_layers = max_layers;
  opt.ignore_components = ignore_components;
  opt.threads = threads < 1 ? 1 : (threads > 64 ? 64 : threads);
  // the stream's sizes drive host allocations: an oversized (or corrupt but well-formed)
  // header fails here with an error code instead of an exception through the C ABI
  int rc;
  try {
    rc = j2k::build_plan(cs, len, opt, p->p);
  } catch (const std::bad_alloc &) {
    delete p;
    return J2K_ERR_NOMEM;
  } catch (...) {
    delete p;
    return J2K_ERR_PARSE;
  }
  if (rc != j2k::PARSE_OK) {
    delete p;
    return rc == j2k::PARSE_ERR_UNSUPPORTED ? J2K_ERR_UNSUPPORTED : J2K_ERR_PARSE;
  }
  *out = p;
  return J2K_OK;
}

extern "C" int j2k_plan_create(const uint8_t *cs, size_t len, int discard_levels, int max_layers,
                               unsigned ignore_components, j2k_plan **out) {
  return j2k_plan_create_mt(cs, len, discard_levels, max_layers, ignore_components, 1, out);
}

extern "C" void j2k_plan_destroy(j2k_plan *p) {
  if (!p) return;
  j2k::give_plan_bytes(std::move(p->p.bytes));
  delete p;
}

extern "C" int j2k_plan_info(const j2k_plan *p, j2k_image_info *info) {
  if (!p || !info) return J2K_ERR_ARG;
  *info = p->p.info;
  return J2K_OK;
}
extern "C" const j2k_cblk *j2k_plan_cblks(const j2k_plan *p) { return p ? p->p.cblks.data() : nullptr; }
extern "C" const uint32_t *j2k_plan_seglens(const j2k_plan *p) { return p ? p->p.seglens.data() : nullptr; }
extern "C" const uint8_t *j2k_plan_bytes(const j2k_plan *p) { return p ? p->p.bytes.data() : nullptr; }
extern "C" const j2k_tilecomp *j2k_plan_tilecomps(const j2k_plan *p) { return p ? p->p.tilecomps.data() : nullptr; }

extern "C" size_t j2k_output_bytes(const j2k_image_info *info, int fmt) {
  if (!info) return 0;
  size_t px = (size_t)info->width * info->height;
  switch (fmt) {
    case J2K_FMT_32BITS_ARGB:
    case J2K_FMT_32BITS_4COMPONENTS: return px * 4;
    case J2K_FMT_48BITS_RGB:
    case J2K_FMT_48BITS_3COMPONENTS: return px * 6;
    case J2K_FMT_24BITS_RGB:
    case J2K_FMT_24BITS_3COMPONENTS: return px * 3;
    case J2K_FMT_64BITS_4COMPONENTS:
    case J2K_FMT_64BITS_ARGB: return px * 8;
    default: return 0;
  }
}

extern "C" const char *j2k_status_string(int s) {
  switch (s) {
    case J2K_OK: return "ok";
    case J2K_ERR_ARG: return "invalid argument";
    case J2K_ERR_PARSE: return "codestream parse error";
    case J2K_ERR_UNSUPPORTED: return "unsupported codestream feature";
    case J2K_ERR_CUDA: return "CUDA error";
    case J2K_ERR_NOMEM: return "device memory budget exceeded";
    case J2K_ERR_TIMEOUT: return "timeout";
    case J2K_ERR_DECODE: return "Tier-1 decode error in at least one code-block";
    case J2K_ERR_STATE: return "invalid call order";
    case J2K_ERR_NODEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}
