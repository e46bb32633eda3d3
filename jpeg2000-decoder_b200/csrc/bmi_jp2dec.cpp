/*
 * bmi_jp2dec.cpp — the reference's C decoding interface (include/bmi_jp2dec.h) on the GPU
 * decode path.
 *
 * Reference behaviour kept (decoder/codec/src/dec_jp2.cpp): BMI_dec_info fills the
 * parameter block from the main header and reports the two pool sizes the caller must
 * allocate (:420-597); BMI_dec_init fails with -1 when a pool is missing or too small
 * (dec_check_param2, :107-137); 0 / -1 return codes; BMI_dec_thumbnail returns PARSING on
 * success (:248-270, :400); BMI_dec_isr is an FPGA stub and BMI_dec_exit releases state.
 * The pools are accounted for but the device pool of the shared context does the work;
 * BMI_dec_init keeps its thread count at the start of pool 0 (the reference keeps its
 * decoder state in that pool), and BMI_dec spreads a multi-tile picture's Tier-2 over
 * that many host threads.
 */
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/bmi_jp2dec.h"
#include "../../include/j2k_gpu.h"
#include "codestream.h"

namespace {
std::mutex g_mu;
j2k_gpu_ctx *g_ctx = nullptr;

// what BMI_dec_init leaves at the start of pool 0
struct InitRecord {
  uint32_t magic;
  int32_t threads;
};
constexpr uint32_t kInitMagic = 0x4A324B54u;

int tier2_threads(const stru_dec_param *p) {
  if (!p->mempool[0] || p->pool_size[0] < (int)sizeof(InitRecord)) return 1;
  InitRecord r;
  std::memcpy(&r, p->mempool[0], sizeof(r));
  return r.magic == kInitMagic && r.threads > 1 ? r.threads : 1;
}

j2k_gpu_ctx *ctx() {
  if (!g_ctx && j2k_gpu_ctx_create(0, 0, &g_ctx) != J2K_OK) g_ctx = nullptr;
  return g_ctx;
}

int decode_planes(stru_dec_param *p, void *output[MAX_COMPONENT], int discard) {
  if (!p || !p->input || p->in_size < 2 || !output) return -1;
  j2k_gpu_ctx *c = ctx();
  if (!c) return -1;
  j2k_plan *plan = nullptr;
  if (j2k_plan_create_mt((const uint8_t *)p->input, p->in_size, discard, 0, 0, tier2_threads(p), &plan) != J2K_OK)
    return -1;
  j2k_image_info I;
  j2k_plan_info(plan, &I);
  // colour pictures come back through the inverse MCT (RGB order), others per component
  const bool rgb = I.ncomp >= 3 && I.mct;
  const bool wide = I.bitdepth > 8;
  const int fmt = rgb ? (wide ? J2K_FMT_48BITS_RGB : J2K_FMT_24BITS_RGB) : J2K_FMT_NONE;
  int rc = -1;
  if (j2k_gpu_batch_begin(c) == J2K_OK && j2k_gpu_batch_add(c, plan, fmt, 0, nullptr) == J2K_OK &&
      j2k_gpu_batch_launch(c, nullptr) == J2K_OK && j2k_gpu_batch_sync(c, -1) == J2K_OK) {
    const size_t n = (size_t)I.width * I.height;
    const int dc = 1 << (I.bitdepth - 1), maxv = (1 << I.bitdepth) - 1;
    rc = j2k_gpu_image_status(c, 0, nullptr) == J2K_OK ? 0 : -1;
    if (rgb) {
      std::vector<uint8_t> px(j2k_output_bytes(&I, fmt));
      if (j2k_gpu_output_copy(c, 0, px.data(), px.size()) != J2K_OK) rc = -1;
      // RGB_24BITS / RGB_48BITS store B, G, R; the container holds the LIFTed value
      for (int comp = 0; comp < 3 && rc == 0; ++comp) {
        if (!output[comp]) continue;
        for (size_t i = 0; i < n; ++i) {
          if (wide) {
            const uint16_t v = reinterpret_cast<const uint16_t *>(px.data())[i * 3 + (2 - comp)];
            ((uint16_t *)output[comp])[i] = (uint16_t)(v >> (16 - I.bitdepth));
          } else {
            ((uint8_t *)output[comp])[i] = px[i * 3 + (2 - comp)];
          }
        }
      }
    } else {
      // each plane on its component's own grid (sub-sampled components are smaller)
      std::vector<int32_t> tmp(n);
      for (int comp = 0; comp < I.ncomp && comp < MAX_COMPONENT && rc == 0; ++comp) {
        if (!output[comp]) continue;
        const size_t nc = (size_t)I.comp_w[comp] * I.comp_h[comp];
        if (j2k_gpu_component_copy(c, 0, comp, tmp.data(), nc * 4) != J2K_OK) {
          rc = -1;
          break;
        }
        for (size_t i = 0; i < nc; ++i) {
          int v = I.reversible ? tmp[i] : (int)reinterpret_cast<const float *>(tmp.data())[i];
          v += dc;
          v = v < 0 ? 0 : (v > maxv ? maxv : v);
          if (!wide) ((uint8_t *)output[comp])[i] = (uint8_t)v;
          else ((uint16_t *)output[comp])[i] = (uint16_t)v;
        }
      }
    }
  }
  j2k_gpu_batch_begin(c);
  j2k_plan_destroy(plan);
  return rc;
}
}  // namespace

extern "C" int BMI_dec_info(stru_dec_param *p, int thread_num) {
  (void)thread_num;
  if (!p || !p->input || p->in_size < 2) return -1;
  j2k::StreamHeader H;
  if (j2k::parse_header((const uint8_t *)p->input, p->in_size, H) != j2k::PARSE_OK) return -1;
  p->width = H.image_w();
  p->height = H.image_h();
  p->bitdepth = H.depth[0];
  p->num_components = H.ncomp;
  p->format = H.ncomp;
  p->cb_width = 1 << H.cbw_exp[0];
  p->cb_height = 1 << H.cbh_exp[0];
  p->prec_width = 1 << H.ppx[0][H.levels[0]];
  p->prec_height = 1 << H.ppy[0][H.levels[0]];
  p->tile_width = H.tile_w;
  p->tile_height = H.tile_h;
  p->tile_num = H.ntx() * H.nty();
  p->layer = H.layers;
  p->dwt_level = H.levels[0];
  p->roi_shift = H.roi_shift[0];
  p->progression = (Jp2_Progression)H.progression;
  p->configuration = (H.cbstyle[0] & 0x3F) | (H.sop ? CONF_SOP : 0) | (H.eph ? CONF_EPH : 0) |
                     (H.reversible[0] ? 0 : (CONF_DWT97 | CONF_QUANT)) | (H.mct ? CONF_MCT : 0) |
                     (H.cs_offset ? CONF_JP2FILE : 0);
  p->guard_bit = H.guard[0];
  for (int i = 0; i <= 3 * MAX_DWT_LEVEL; ++i) p->quant_step[i] = H.steps[0][i];
  // pool 0: host Tier-2 state; pool 1: one decoded picture (4 bytes per sample)
  const size_t samples = (size_t)H.image_w() * H.image_h() * H.ncomp;
  p->pool_size[0] = (int)std::min<size_t>(0x7FFFFFFF, p->in_size + samples / 16 + 4096);
  p->pool_size[1] = (int)std::min<size_t>(0x7FFFFFFF, samples * 4);
  p->size_opt = 0;
  return 0;
}

extern "C" int BMI_dec_init(stru_dec_param *p, int use_j2k_header, int thread_num) {
  (void)use_j2k_header;
  if (!p) return -1;
  if (!p->mempool[0] || !p->mempool[1] || p->pool_size[0] < (int)sizeof(InitRecord) || p->pool_size[1] <= 0)
    return -1;
  const InitRecord r{kInitMagic, thread_num > 1 ? thread_num : 1};
  std::memcpy(p->mempool[0], &r, sizeof(r));
  std::lock_guard<std::mutex> g(g_mu);
  return ctx() ? 0 : -1;
}

extern "C" int BMI_dec_isr(stru_dec_param *p, int fpga_irq) {
  (void)p;
  (void)fpga_irq;
  return 0;
}

extern "C" int BMI_dec(stru_dec_param *p, void *output[MAX_COMPONENT], int use_j2k_header) {
  (void)use_j2k_header;
  std::lock_guard<std::mutex> g(g_mu);
  return decode_planes(p, output, 0);
}

extern "C" BMI::Status BMI_dec_thumbnail(stru_dec_param *p, void *output[MAX_COMPONENT], int resolution,
                                         int use_j2k_header) {
  (void)use_j2k_header;
  std::lock_guard<std::mutex> g(g_mu);
  if (!p || !p->input) return BMI::PARSE_ERROR_INVALID_INPUT;
  return decode_planes(p, output, resolution < 0 ? 0 : resolution) == 0 ? BMI::PARSING : BMI::PARSE_ERROR;
}

extern "C" int BMI_dec_exit(stru_dec_param *p) {
  (void)p;
  std::lock_guard<std::mutex> g(g_mu);
  if (g_ctx) j2k_gpu_ctx_destroy(g_ctx);
  g_ctx = nullptr;
  return 0;
}
