/*
 * engine.cu — device context, batching and the j2k_gpu C ABI (include/j2k_gpu.h).
 *
 * A batch is a set of decode plans.  batch_launch concatenates their Tier-1 work lists,
 * coded bytes and DWT/output task tables into one pinned staging area, copies each
 * section to the device with one cudaMemcpyAsync, then enqueues:
 *   - Tier-1: a persistent launch that drains a work queue sorted by coded length (longest
 *     first), one code-block per warp (t1_kernel.cuh); on request (t1_form 3) one block per
 *     lane (t1_lanes.cuh) for blocks up to 64x64 without bypass segments;
 *   - inverse DWT: one launch per level step for all tile-components of all images
 *     (5/3 and 9/7 variants), coarsest level first;
 *   - inverse MCT + DC shift + pack into each image's output;
 *   - the per-block status back to the host.
 * This replaces the reference's CudaManager job thread with its per-stripe H2D copies and
 * per-component launch sequence (decoder/cudainterface/src/cudainterface.cpp:1072-1765,
 * :2276-2640, gpulib.c:165-343).  There is no CPU fallback: without a device every call
 * fails with J2K_ERR_NODEVICE.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <new>
#include <thread>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/j2k_gpu.h"
#include "bmi_engine.h"
#include "codestream.h"
#include "dwt_kernel.cuh"
#include "t1_kernel.cuh"
#include "t1_lanes.cuh"

using namespace j2k_dev;

namespace {

// ------------------------------------------------------------------ Tier-1 kernel -------
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

template <int MAXW, int MAXH>
struct T1Layout {
  static constexpr int STRIPES = MAXH / 4;
  static constexpr int GAP = MAXW + 3;
  static constexpr int CWN = (STRIPES + 2) * GAP + 2;
  static constexpr int RF_BYTES = ((STRIPES * GAP) + 3) & ~3;
  // context words, refined bits, MQ context slots, then 32 bytes of per-chunk row masks
  static constexpr int PER_WARP = ((CWN * 4 + RF_BYTES + N_CTX * 8 + 32) + 15) & ~15;
};

// Host-side queue classes: blocks the lane form decodes (up to 64x64, no bypass segments;
// filled only when the batch is staged with t1_form 3) and the others; the warp forms take
// both, as one queue (the two are contiguous), so without the lane form it is one queue
// sorted longest first.
enum { QL = 0, QW = 1, NQ = 2 };
// The warp forms' tables (MQ states, zero-coding / sign contexts, bypass refinement
// scatter) in constant memory: every lane of a warp reads the same entry, so the constant
// cache broadcasts it, and the loads need no shared-memory copy per CTA.
__constant__ T1Tables c_t1tables;

template <int MAXW, int MAXH, bool UNROLLED>
__device__ __forceinline__ void t1_body(const j2k_cblk *__restrict__ cbs, const uint32_t *__restrict__ order, int n,
                                        int *__restrict__ counter, const uint8_t *__restrict__ bytes,
                                        const uint32_t *__restrict__ seglens, void *__restrict__ coef,
                                        uint16_t *__restrict__ status) {
  extern __shared__ __align__(16) uint8_t smem[];
  typedef T1Layout<MAXW, MAXH> Lay;
  const T1Tables &T = c_t1tables;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t *mine = smem + warp * Lay::PER_WARP;
  BlockSmem b;
  b.cw = reinterpret_cast<uint32_t *>(mine);
  b.rf = mine + Lay::CWN * 4;
  b.cx = reinterpret_cast<uint2 *>(mine + Lay::CWN * 4 + Lay::RF_BYTES);
  b.sp.lane = lane;
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(counter, 1);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= n) break;
    const uint32_t ci = order[idx];
    const j2k_cblk cb = cbs[ci];
    b.w = cb.w;
    b.gap = cb.w + 3;
    int32_t *blk = reinterpret_cast<int32_t *>(coef) + cb.out_off;
    b.sp.base = blk;
    b.sp.stride = cb.out_stride;
    int bit_plane, num_passes;
    block_planes(cb, bit_plane, num_passes);
    int st;
    if (cb.w == 0 || cb.h == 0 || cb.w > MAXW || cb.h > MAXH) {
      st = 9;
    } else {
      st = decode_block<UNROLLED>(cb, bytes, seglens, b, T, lane, bit_plane, num_passes);
    }
    // rewrite the block in place: raw sign-magnitude -> dequantised float (9/7) or shifted
    // integer (5/3); the lanes' sample writes are made visible first.  A sample whose
    // significance bit (context word, shared memory) is clear was never written: it is 0.
    const int w = cb.w, h = cb.h;
    if (st != 9) {
      __threadfence();
      __syncwarp();
      const bool irrev = (cb.flags & J2K_CB_IRREV) != 0;
      for (int y = 0; y < h; ++y) {
        int32_t *r = blk + (size_t)y * cb.out_stride;
        const uint32_t sig = ROW_SIG(y & 3);
        const uint32_t *wrow = cword(b, y >> 2, 0);
        for (int x = lane; x < w; x += 32) {
          const int32_t v = (wrow[x] & sig) ? __ldcg(r + x) : 0;
          if (irrev) *reinterpret_cast<float *>(r + x) = __fmul_rn((float)signmag_to_int(v), cb.gain);
          else r[x] = place53(v, cb.mb);
        }
      }
    }
    if (lane == 0) status[ci] = (uint16_t)st;
    __syncwarp();
  }
}

// The two kernel forms.  The compact form keeps the default register target, which leaves
// room for 32 resident warps per SM; the unrolled form (batches that fit one wave) may use
// more registers, as occupancy does not bound it.
#define J2K_T1_PARAMS                                                                                   \
  const j2k_cblk *__restrict__ cbs, const uint32_t *__restrict__ order, int n, int *__restrict__ counter, \
      const uint8_t *__restrict__ bytes, const uint32_t *__restrict__ seglens, void *__restrict__ coef,   \
      uint16_t *__restrict__ status
template <int MAXW, int MAXH>
__global__ void __launch_bounds__(256) t1_kernel_compact(J2K_T1_PARAMS) {
  t1_body<MAXW, MAXH, false>(cbs, order, n, counter, bytes, seglens, coef, status);
}
template <int MAXW, int MAXH>
__global__ void __launch_bounds__(256, 1) t1_kernel_unrolled(J2K_T1_PARAMS) {
  t1_body<MAXW, MAXH, true>(cbs, order, n, counter, bytes, seglens, coef, status);
}
#undef J2K_T1_PARAMS

template <int MAXW, int MAXH, bool UNROLLED>
constexpr auto t1_kernel() {
  if constexpr (UNROLLED) return &t1_kernel_unrolled<MAXW, MAXH>;
  else return &t1_kernel_compact<MAXW, MAXH>;
}

// ------------------------------------------------------------------ host tables --------
void build_t1_tables(T1Tables &T) {
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
  std::memset(&T, 0, sizeof(T));
  for (int s = 0; s < 94; ++s) {
    int idx = s >> 1, mps = s & 1;
    int sw = (QE[idx] == 0x5601 && NLPS[idx] != 46);
    uint32_t nm = (uint32_t)(NMPS[idx] << 1 | mps);
    uint32_t nl = (uint32_t)(NLPS[idx] << 1 | (mps ^ sw));
    T.mq[s].x = (uint32_t)QE[idx] << 8;
    T.mq[s].y = ((uint32_t)mps << 16) | (nm << 8) | nl;
  }
  for (int r = 0; r < 16; ++r) {
    const int n = __builtin_popcount(r);
    for (int x = 0; x < (1 << n); ++x) {
      int v = 0, i = 0;
      for (int k = 0; k < 4; ++k)
        if ((r >> k) & 1) v |= ((x >> (n - 1 - i++)) & 1) << k;
      T.rawmr[r][x] = (uint8_t)v;
    }
  }
  for (int band = 0; band < 3; ++band)
    for (int nb = 0; nb < 512; ++nb) {
      int h = ((nb >> 3) & 1) + ((nb >> 5) & 1);
      int v = ((nb >> 1) & 1) + ((nb >> 7) & 1);
      int d = (nb & 1) + ((nb >> 2) & 1) + ((nb >> 6) & 1) + ((nb >> 8) & 1);
      int c;
      if (band == 2) {  // HH
        int hv = h + v;
        if (d >= 3) c = 8;
        else if (d == 2) c = hv >= 1 ? 7 : 6;
        else if (d == 1) c = hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
        else c = hv >= 2 ? 2 : hv;
      } else {
        if (band == 1) std::swap(h, v);  // HL
        if (h == 2) c = 8;
        else if (h == 1) c = v >= 1 ? 7 : (d >= 1 ? 6 : 5);
        else if (v == 2) c = 4;
        else if (v == 1) c = 3;
        else c = d >= 2 ? 2 : d;
      }
      T.zc[band][nb] = (uint8_t)c;
    }
  for (int i = 0; i < 256; ++i) {
    // bit 0 sigma up, 1 chi up, 2 sigma down, 3 chi down, 4 sigma left, 5 chi left,
    // 6 sigma right, 7 chi right (T.800 Table D.3)
    auto contrib = [&](int sb, int xb) { return ((i >> sb) & 1) ? (((i >> xb) & 1) ? -1 : 1) : 0; };
    int H = contrib(4, 5) + contrib(6, 7);
    int V = contrib(0, 1) + contrib(2, 3);
    H = std::max(-1, std::min(1, H));
    V = std::max(-1, std::min(1, V));
    int x = 0;
    if (H < 0 || (H == 0 && V < 0)) {
      H = -H;
      V = -V;
      x = 1;
    }
    int c = (H == 1) ? (V == 1 ? 4 : (V == 0 ? 3 : 2)) : (V == 1 ? 1 : 0);
    T.sc[i] = (uint8_t)(c << 1 | x);
  }
}

// ------------------------------------------------------------------ device buffers -----
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
};

struct BatchImage {
  const j2k_plan *plan;
  int fmt, flags;
  int checkout;
  uint64_t coef_base, out_base, out_bytes;
  uint32_t cblk_base;
  int status, bad;
  bool fused;  // last DWT level fused with the output stage: components not kept
};

}  // namespace

struct j2k_gpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr, user_stream = nullptr;
  size_t budget = 0, reserved = 0;
  DevBuf d_bytes, d_cblks, d_order, d_seg, d_status, d_counter, d_A, d_B, d_C, d_levels, d_dtasks, d_groups, d_otasks,
      d_out, d_tables;
  void *h_stage = nullptr;
  size_t h_stage_cap = 0;
  std::vector<BatchImage> imgs;
  uint16_t *h_status = nullptr;  // pinned
  size_t h_status_cap = 0;
  // outgrown pinned staging / status areas: freeing page-locked memory waits for the whole
  // device, which would stall other contexts' work in flight, so they go at ctx_destroy
  std::vector<void *> h_retired;
  bool launched = false, synced = false, staged = false;
  bool copies_pending = false;  // output copies enqueued behind the decode (ev[5] follows them)
  // staged batch (device-resident inputs) for batch_run
  struct Staged {
    size_t nq[NQ] = {0}, n_cblks = 0, n_otasks = 0;
    size_t o_cbs = 0, o_ord = 0, o_seg = 0, o_lev = 0, o_dtk = 0, o_grp = 0, o_otk = 0, o_fgr = 0, o_ftk = 0;
    size_t n_ftasks[2] = {0, 0};
    size_t o_ctk = 0, n_ctasks[2] = {0, 0};  // coarse-level tasks: [0] 9/7, [1] 5/3
    int fwin = 1;
    int maxL = 0;
    std::vector<uint32_t> dtask_off;
  } sg;
  cudaEvent_t ev[6] = {};  // h2d start, h2d end, Tier-1 end, DWT end, decode end, output copies end
  float t_t1 = 0, t_dwt = 0, t_h2d = 0, t_total = 0;
  int launches = 0;
  j2k_gpu_tuning tuning{8, 64, 0, 0, 2, 0};
  cudaGraphExec_t gexec = nullptr;  // captured decode of the staged batch (tuning.use_graph)
  int graph_launches = 0;
  // autotuned Tier-1 shape per queue-length bucket (floor(log2(code-blocks))): kernel form
  // (1 compact, 2 unrolled) and warps per CTA; consulted by the auto form
  struct TuneEntry {
    int form = 0, warps = 0;
    float t1_ms = 0;
  };
  std::map<int, TuneEntry> tune_table;
  int dwt_auto = 0;  // autotuned coarse-level choice (1 on, 2 off) for dwt_coarse 0; 0 = not tuned (on)
  int sm_count = 148;
  size_t smem_optin = 227 * 1024;
};

namespace {

void drop_graph(j2k_gpu_ctx *c) {
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  c->gexec = nullptr;
}

int cuda_fail(cudaError_t e) {
  (void)e;
  return J2K_ERR_CUDA;
}

#define CK(x)                                  \
  do {                                         \
    cudaError_t _e = (x);                      \
    if (_e != cudaSuccess) return cuda_fail(_e); \
  } while (0)

int ensure(j2k_gpu_ctx *c, DevBuf &b, size_t need) {
  if (need == 0) need = 16;
  if (b.cap >= need) return J2K_OK;
  // grow to twice the old size at least (within the budget): replacing a device buffer
  // frees the old one, which waits for the whole device, and allocating gigabytes takes
  // hundreds of milliseconds, so a pool warmed on a stream of mixed batches should not have
  // to grow again for a batch a little larger than the ones it has seen
  size_t nc = std::max(need, b.cap * 2);
  if (c->reserved - b.cap + nc > c->budget) {
    nc = need;
    if (c->reserved - b.cap + nc > c->budget) return J2K_ERR_NOMEM;
  }
  if (b.p) {
    cudaFree(b.p);
    c->reserved -= b.cap;
    b.p = nullptr;
    b.cap = 0;
  }
  cudaError_t e = cudaMalloc(&b.p, nc);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return J2K_ERR_NOMEM;
  }
  b.cap = nc;
  c->reserved += nc;
  return J2K_OK;
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace

extern "C" int j2k_gpu_ctx_create(int device, size_t mem_budget, j2k_gpu_ctx **out) {
  if (!out) return J2K_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return J2K_ERR_NODEVICE;
  }
  if (device < 0 || device >= n) return J2K_ERR_ARG;
  j2k_gpu_ctx *c = new (std::nothrow) j2k_gpu_ctx;
  if (!c) return J2K_ERR_NOMEM;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete c;
    return J2K_ERR_CUDA;
  }
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  c->budget = mem_budget ? mem_budget : (size_t)(fr * 0.8);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
    c->sm_count = prop.multiProcessorCount;
    c->smem_optin = prop.sharedMemPerBlockOptin;
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return J2K_ERR_CUDA;
  }
  for (auto &e : c->ev) cudaEventCreate(&e);
  T1Tables T;
  build_t1_tables(T);
  j2k_lanes::LaneTables LT;
  j2k_lanes::build_lane_tables(LT);
  if (cudaMemcpyToSymbol(c_t1tables, &T, sizeof(T)) != cudaSuccess || ensure(c, c->d_tables, sizeof(LT)) != J2K_OK ||
      cudaMemcpy(c->d_tables.p, &LT, sizeof(LT), cudaMemcpyHostToDevice) != cudaSuccess) {
    j2k_gpu_ctx_destroy(c);
    return J2K_ERR_CUDA;
  }
  // opt into the large dynamic shared memory of the Tier-1 kernels
  if (j2k_lanes::CTA_SMEM <= c->smem_optin)
    cudaFuncSetAttribute(j2k_lanes::t1_kernel_lanes, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)j2k_lanes::CTA_SMEM);
  cudaFuncSetAttribute(t1_kernel<64, 64, false>(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem_optin);
  cudaFuncSetAttribute(t1_kernel<64, 64, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem_optin);
  cudaFuncSetAttribute(last_level_output_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(3 * sizeof(DwtSmem<true>)));
  cudaFuncSetAttribute(last_level_output_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(3 * sizeof(DwtSmem<false>)));
  *out = c;
  return J2K_OK;
}

extern "C" void j2k_gpu_ctx_destroy(j2k_gpu_ctx *c) {
  if (!c) return;
  drop_graph(c);
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  DevBuf *all[] = {&c->d_bytes, &c->d_cblks, &c->d_order, &c->d_seg,    &c->d_status, &c->d_counter,
                   &c->d_A,     &c->d_B,     &c->d_C,     &c->d_levels, &c->d_dtasks, &c->d_groups,
                   &c->d_otasks, &c->d_out,  &c->d_tables};
  for (DevBuf *b : all)
    if (b->p) cudaFree(b->p);
  if (c->h_stage) cudaFreeHost(c->h_stage);
  if (c->h_status) cudaFreeHost(c->h_status);
  for (void *p : c->h_retired) cudaFreeHost(p);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" int j2k_gpu_mem_usage(const j2k_gpu_ctx *c, size_t *reserved, size_t *budget) {
  if (!c) return J2K_ERR_ARG;
  if (reserved) *reserved = c->reserved;
  if (budget) *budget = c->budget;
  return J2K_OK;
}

extern "C" int j2k_gpu_set_tuning(j2k_gpu_ctx *c, const j2k_gpu_tuning *t) {
  if (!c || !t) return J2K_ERR_ARG;
  j2k_gpu_tuning n = *t;
  if (n.t1_warps_per_cta <= 0) n.t1_warps_per_cta = 8;
  if (n.t1_warps_per_cta > 32) n.t1_warps_per_cta = 32;
  if (n.dwt_tile <= 0) n.dwt_tile = 64;
  if (n.dwt_tile != 64) return J2K_ERR_UNSUPPORTED;  // the level kernels are built for 64x64 tiles
  if (n.t1_form < 0 || n.t1_form > 3) n.t1_form = 0;
  if (n.t1_latency_waves <= 0) n.t1_latency_waves = 2;
  if (n.dwt_coarse < 0 || n.dwt_coarse > 2) n.dwt_coarse = 0;  // takes effect at the next batch_stage
  if (n.use_graph != c->tuning.use_graph || n.t1_form != c->tuning.t1_form || n.dwt_coarse != c->tuning.dwt_coarse ||
      n.t1_warps_per_cta != c->tuning.t1_warps_per_cta || n.t1_latency_waves != c->tuning.t1_latency_waves)
    drop_graph(c);
  c->tuning = n;
  return J2K_OK;
}
extern "C" int j2k_gpu_get_tuning(const j2k_gpu_ctx *c, j2k_gpu_tuning *t) {
  if (!c || !t) return J2K_ERR_ARG;
  *t = c->tuning;
  return J2K_OK;
}

extern "C" int j2k_gpu_batch_begin(j2k_gpu_ctx *c) {
  if (!c) return J2K_ERR_ARG;
  if (c->launched && !c->synced) return J2K_ERR_STATE;
  c->imgs.clear();
  c->launched = c->synced = c->staged = c->copies_pending = false;
  return J2K_OK;
}

extern "C" int j2k_gpu_batch_add(j2k_gpu_ctx *c, const j2k_plan *plan, int fmt, int flags, int *slot) {
  if (!c || !plan) return J2K_ERR_ARG;
  if (c->launched || c->staged) return J2K_ERR_STATE;
  if (fmt != J2K_FMT_NONE && j2k_dev::fmt_bytes(fmt) == 0) return J2K_ERR_ARG;
  const j2k_image_info &I = plan->p.info;
  if (I.bitdepth < 1 || I.bitdepth > 16) return J2K_ERR_UNSUPPORTED;
  // packed pictures are laid on component 0's grid: it must be the picture grid
  if (fmt != J2K_FMT_NONE && (I.sub_x[0] != 1 || I.sub_y[0] != 1)) return J2K_ERR_UNSUPPORTED;
  BatchImage bi{};
  bi.checkout = -1;
  bi.plan = plan;
  bi.fmt = fmt;
  bi.flags = flags;
  if (slot) *slot = (int)c->imgs.size();
  c->imgs.push_back(bi);
  return J2K_OK;
}

namespace {

struct Sizes {
  size_t bytes = 0, cblks = 0, segs = 0, coef = 0, out = 0;
};

Sizes batch_sizes(j2k_gpu_ctx *c) {
  Sizes s;
  for (auto &im : c->imgs) {
    const auto &p = im.plan->p;
    im.coef_base = s.coef;
    im.cblk_base = (uint32_t)s.cblks;
    im.out_base = align_up(s.out, 256);
    im.out_bytes = im.fmt == J2K_FMT_NONE ? 0 : j2k_output_bytes(&p.info, im.fmt);
    s.bytes += p.bytes.size();
    s.cblks += p.cblks.size();
    s.segs += p.seglens.size();
    s.coef += p.info.coef_elems;
    s.out = im.out_base + im.out_bytes;
  }
  return s;
}

}  // namespace

extern "C" int j2k_gpu_batch_footprint(const j2k_gpu_ctx *cc, size_t *bytes) {
  if (!cc || !bytes) return J2K_ERR_ARG;
  j2k_gpu_ctx *c = const_cast<j2k_gpu_ctx *>(cc);
  Sizes s = batch_sizes(c);
  *bytes = s.bytes + s.cblks * (sizeof(j2k_cblk) + 4 + 2) + s.segs * 4 + s.coef * 12 + s.out;
  return J2K_OK;
}

namespace {
// Persistent Tier-1 launch: the CTA shape with the most resident warps per SM (registers,
// shared memory and thread limits from the occupancy calculator), one wave of CTAs.
template <int MAXW, int MAXH, bool UNROLLED>
void launch_t1_as(j2k_gpu_ctx *c, cudaStream_t st, int n, const j2k_cblk *cbs, const uint32_t *ord, int *cnt,
                  const uint32_t *seg, int warps_per_cta) {
  typedef T1Layout<MAXW, MAXH> Lay;
  int best_w = 1, best_ctas = 1, best_warps = 0;
  const int wmax = warps_per_cta > 0 ? std::min(8, warps_per_cta) : 8;
  for (int w = 1; w <= wmax; ++w) {
    const size_t sm = (size_t)w * Lay::PER_WARP;
    if (sm > c->smem_optin) break;
    int ctas = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas, t1_kernel<MAXW, MAXH, UNROLLED>(), w * 32, sm) !=
        cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (ctas * w > best_warps || (ctas * w == best_warps && w > best_w)) {
      best_warps = ctas * w;
      best_w = w;
      best_ctas = ctas;
    }
  }
  const size_t sm = (size_t)best_w * Lay::PER_WARP;
  const int grid = std::max(1, std::min((n + best_w - 1) / best_w, c->sm_count * std::max(1, best_ctas)));
  t1_kernel<MAXW, MAXH, UNROLLED>()<<<grid, best_w * 32, sm, st>>>(cbs, ord, n, cnt, (const uint8_t *)c->d_bytes.p, seg,
                                                                     c->d_A.p, (uint16_t *)c->d_status.p);
}

// Tier-1 form for a batch of n code-blocks: 1 compact warp form (throughput), 2 unrolled
// warp form (latency), 3 one block per lane, and warps per CTA of a warp form.  An explicit
// tuning.t1_form wins; the auto form (0) takes the autotuned choice of the queue's size
// bucket, else the unrolled form while the queue holds at most `t1_latency_waves` blocks
// per resident warp slot of the GPU (the launch's time is then the serial time of its
// longest blocks) and the compact form for longer queues.  The lane form is only taken
// when asked for: on B200 it measured 4.2x slower than the compact form on 1080p 9/7
// frames (its lanes' pass walks diverge: 4.4 of 32 threads active per instruction).
void t1_shape(const j2k_gpu_ctx *c, int n, int &form, int &warps) {
  warps = c->tuning.t1_warps_per_cta;
  if (c->tuning.t1_form >= 1 && c->tuning.t1_form <= 3) {
    form = c->tuning.t1_form;
    return;
  }
  auto it = c->tune_table.find(n > 0 ? 31 - __builtin_clz((unsigned)n) : 0);
  if (it != c->tune_table.end()) {
    form = it->second.form;
    warps = it->second.warps;
    return;
  }
  const int waves = c->tuning.t1_latency_waves > 0 ? c->tuning.t1_latency_waves : 2;
  form = (long long)n <= (long long)waves * c->sm_count * 32 ? 2 : 1;
}

// Enqueue the Tier-1 stage: the lane kernel on the lane queue and a warp form on the rest,
// or a warp form on both queues (contiguous in `ord`).  Returns the number of launches.
int launch_t1(j2k_gpu_ctx *c, cudaStream_t st, const size_t nq[NQ], const j2k_cblk *cbs, const uint32_t *ord,
              int *cnt, const uint32_t *seg, const j2k_lanes::LaneTables *ltab) {
  const int nl = (int)nq[QL], nw = (int)nq[QW], n = nl + nw;
  if (!n) return 0;
  int form, warps;
  t1_shape(c, n, form, warps);
  const bool lanes_ok = j2k_lanes::CTA_SMEM <= c->smem_optin;
  if (form == 3 && nl > 0 && lanes_ok) {
    const int grid = std::max(1, std::min(c->sm_count, nl));
    j2k_lanes::t1_kernel_lanes<<<grid, j2k_lanes::CTA_WARPS * 32, j2k_lanes::CTA_SMEM, st>>>(
        cbs, ord, nl, cnt, (const uint8_t *)c->d_bytes.p, seg, c->d_A.p, (uint16_t *)c->d_status.p, ltab);
    if (!nw) return 1;
    launch_t1_as<64, 64, false>(c, st, nw, cbs, ord + nl, cnt + 1, seg, warps);
    return 2;
  }
  if (form == 3) form = 1;  // no lane-form blocks (or too little shared memory): compact warp form
  if (form == 2) launch_t1_as<64, 64, true>(c, st, n, cbs, ord, cnt, seg, warps);
  else launch_t1_as<64, 64, false>(c, st, n, cbs, ord, cnt, seg, warps);
  return 1;
}
}  // namespace

extern "C" int j2k_gpu_batch_stage(j2k_gpu_ctx *c, void *user_stream) {
  if (!c) return J2K_ERR_ARG;
  if (c->launched && !c->synced) return J2K_ERR_STATE;
  if (c->imgs.empty()) return J2K_ERR_STATE;
  cudaSetDevice(c->device);
  cudaStream_t st = user_stream ? (cudaStream_t)user_stream : c->stream;
  c->user_stream = st;
  Sizes S = batch_sizes(c);

  // ---- host task tables
  std::vector<j2k_cblk> cbs;
  cbs.reserve(S.cblks);
  std::vector<uint32_t> seg;
  seg.reserve(S.segs);
  std::vector<uint32_t> ordq[NQ];
  std::vector<DwtLevel> levels;
  std::vector<std::vector<DwtTask>> steps_rev, steps_irr;
  std::vector<OutGroup> groups;
  std::vector<OutTask> otasks;
  std::vector<FusedGroup> fgroups;
  std::vector<OutTask> ftasks[2];  // fused last levels: [0] 9/7, [1] 5/3
  std::vector<CoarseTask> ctasks[2];  // coarse levels synthesised in shared memory: [0] 9/7, [1] 5/3
  const bool coarse_on = c->tuning.dwt_coarse == 1 || (c->tuning.dwt_coarse == 0 && c->dwt_auto != 2);
  const bool lane_split = c->tuning.t1_form == 3;  // queue classes for the lane form
  int fwin = 1;
  uint64_t byte_base = 0;
  uint32_t seg_base = 0;
  int maxL = 0;
  for (auto &im : c->imgs)
    for (auto &tc : im.plan->p.tilecomps) maxL = std::max(maxL, tc.levels);
  steps_rev.resize(maxL);
  steps_irr.resize(maxL);
  for (auto &im : c->imgs) {
    const auto &p = im.plan->p;
    for (const j2k_cblk &cb0 : p.cblks) {
      j2k_cblk cb = cb0;
      cb.data_off = (uint32_t)(cb.data_off + byte_base);
      cb.seg_off += seg_base;
      cb.out_off += im.coef_base;
      uint32_t idx = (uint32_t)cbs.size();
      cbs.push_back(cb);
      ordq[lane_split && j2k_lanes::lane_eligible(cb) ? QL : QW].push_back(idx);
    }
    seg.insert(seg.end(), p.seglens.begin(), p.seglens.end());
    byte_base += p.bytes.size();
    seg_base += (uint32_t)p.seglens.size();
    const bool rev = p.info.reversible != 0;
    const int refc = (im.flags & J2K_FLAG_REF_COMPAT) ? 1 : 0;
    // Tiles whose last level is fused with the output stage: packed output wanted, no
    // component kept for the getters, 1-3 components of one size, all with >= 1 level
    std::vector<char> fuse(p.tilecomps.size(), 0);
    im.fused = false;
    if (im.fmt != J2K_FMT_NONE && im.checkout < 0 && !(im.flags & J2K_FLAG_KEEP_COMPONENTS)) {
      for (size_t t = 0; t < p.tilecomps.size(); ++t) {
        const j2k_tilecomp &tc = p.tilecomps[t];
        if (tc.comp != 0) continue;
        bool ok = tc.levels >= 1;
        int nc = 0;
        for (size_t u = 0; u < p.tilecomps.size() && ok; ++u) {
          const j2k_tilecomp &tu = p.tilecomps[u];
          if (tu.tile != tc.tile) continue;
          nc++;
          ok = tu.comp < 3 && tu.levels == tc.levels && tu.w == tc.w && tu.h == tc.h &&
               p.info.sub_x[tu.comp] == 1 && p.info.sub_y[tu.comp] == 1;
        }
        if (!ok || nc < 1 || nc > 3) continue;
        for (size_t u = 0; u < p.tilecomps.size(); ++u)
          if (p.tilecomps[u].tile == tc.tile) fuse[u] = 1;
        im.fused = true;
      }
    }
    // DWT levels of every tile-component, aligned so that all finish at the last step; the
    // coarse levels (every resolution up to COARSE_MAX samples a side, below a fused last
    // level) go to one shared-memory kernel instead
    std::vector<int8_t> final_buf(p.tilecomps.size());
    for (size_t t = 0; t < p.tilecomps.size(); ++t) {
      const j2k_tilecomp &tc = p.tilecomps[t];
      const int Lt = tc.levels;
      final_buf[t] = Lt == 0 ? 0 : ((Lt & 1) ? 1 : 2);
      int rc = 0;
      if (coarse_on) {
        const int top = std::min(fuse[t] ? Lt - 1 : Lt, 7);
        while (rc < top && tc.res_w[rc + 1] <= COARSE_MAX && tc.res_h[rc + 1] <= COARSE_MAX) ++rc;
        if (rc >= 1) {
          CoarseTask ck{};
          ck.base = im.coef_base + tc.coef_off;
          ck.stride = tc.w;
          ck.rc = (int8_t)rc;
          ck.out_dst = (int8_t)((rc & 1) ? 1 : 2);
          ck.refcompat = (int8_t)refc;
          for (int r = 0; r <= rc; ++r) {
            ck.res_w[r] = (int16_t)tc.res_w[r];
            ck.res_h[r] = (int16_t)tc.res_h[r];
          }
          ctasks[rev ? 1 : 0].push_back(ck);
        }
      }
      for (int r = rc + 1; r <= Lt; ++r) {
        DwtLevel L{};
        L.base = im.coef_base + tc.coef_off;
        L.stride = tc.w;
        L.rw = tc.res_w[r];
        L.rh = tc.res_h[r];
        L.lw = tc.res_w[r - 1];
        L.lh = tc.res_h[r - 1];
        L.ll_src = r == 1 ? 0 : (((r - 1) & 1) ? 1 : 2);
        L.out_dst = (r & 1) ? 1 : 2;
        L.ll_gain = (!rev && r > 1) ? 1 : 0;
        L.refcompat = (int8_t)refc;
        if (L.rw <= 0 || L.rh <= 0) continue;
        if (r == Lt && fuse[t]) continue;  // rebuilt by the fused output stage
        L.tiles_x = (L.rw + DWT_T - 1) / DWT_T;
        const int tiles_y = (L.rh + DWT_T - 1) / DWT_T;
        const uint32_t li = (uint32_t)levels.size();
        levels.push_back(L);
        const int step = maxL - Lt + r - 1;
        auto &dst = rev ? steps_rev[step] : steps_irr[step];
        for (int ty = 0; ty < tiles_y; ++ty)
          for (int tx = 0; tx < L.tiles_x; ++tx) dst.push_back({li, (uint16_t)tx, (uint16_t)ty});
      }
    }
    if (im.fmt != J2K_FMT_NONE) {
      // output groups: one per tile
      for (size_t t = 0; t < p.tilecomps.size(); ++t) {
        const j2k_tilecomp &tc = p.tilecomps[t];
        if (tc.comp != 0) continue;
        if (fuse[t]) {
          FusedGroup F{};
          OutGroup &G = F.G;
          for (int k = 0; k < 4; ++k) G.comp_buf[k] = -1;
          int nc = 0;
          const int Lt = tc.levels;
          for (size_t u = 0; u < p.tilecomps.size(); ++u) {
            const j2k_tilecomp &tu = p.tilecomps[u];
            if (tu.tile != tc.tile) continue;
            F.base[tu.comp] = im.coef_base + tu.coef_off;
            F.ll_src[tu.comp] = Lt == 1 ? 0 : (((Lt - 1) & 1) ? 1 : 2);
            G.comp_buf[tu.comp] = 0;
            G.stride[tu.comp] = tu.w;
            nc = std::max(nc, tu.comp + 1);
          }
          F.ll_gain = (!rev && Lt > 1) ? 1 : 0;
          F.refcompat = (int8_t)refc;
          F.stride = tc.w;
          F.rw = tc.res_w[Lt];
          F.rh = tc.res_h[Lt];
          F.lw = tc.res_w[Lt - 1];
          F.lh = tc.res_h[Lt - 1];
          G.x0 = tc.x0;
          G.y0 = tc.y0;
          G.w = tc.w;
          G.h = tc.h;
          G.out_off = im.out_base;
          G.pitch_px = p.info.width;
          G.fmt = (int16_t)im.fmt;
          G.bitdepth = (int16_t)p.info.bitdepth;
          G.rev = (int8_t)rev;
          G.mct = (int8_t)p.info.mct;
          G.ncomp = (int8_t)nc;
          G.checkout = -1;
          G.tiles_x = (tc.w + DWT_T - 1) / DWT_T;
          fwin = std::max(fwin, nc);
          const uint32_t gi = (uint32_t)fgroups.size();
          fgroups.push_back(F);
          for (int ty = 0; ty < (tc.h + DWT_T - 1) / DWT_T; ++ty)
            for (int tx = 0; tx < G.tiles_x; ++tx) ftasks[rev ? 1 : 0].push_back({gi, (uint16_t)tx, (uint16_t)ty});
          continue;
        }
        OutGroup G{};
        for (int k = 0; k < 4; ++k) G.comp_buf[k] = -1;
        int nc = 0;
        G.ax = p.info.origin_x + tc.x0;
        G.ay = p.info.origin_y + tc.y0;
        for (size_t u = 0; u < p.tilecomps.size(); ++u) {
          const j2k_tilecomp &tu = p.tilecomps[u];
          if (tu.tile != tc.tile || tu.comp >= 4) continue;
          G.comp_off[tu.comp] = im.coef_base + tu.coef_off;
          G.comp_buf[tu.comp] = final_buf[u];
          G.stride[tu.comp] = tu.w;
          nc = std::max(nc, tu.comp + 1);
          // component sampling: the tile-component's absolute origin and size on its grid
          const int k = tu.comp;
          G.sx[k] = (uint8_t)p.info.sub_x[k];
          G.sy[k] = (uint8_t)p.info.sub_y[k];
          G.cx[k] = p.info.comp_x0[k] + tu.x0;
          G.cy[k] = p.info.comp_y0[k] + tu.y0;
          G.cw[k] = tu.w;
          G.ch[k] = tu.h;
          if (G.sx[k] != 1 || G.sy[k] != 1) G.sampled = 1;
        }
        G.x0 = tc.x0;
        G.y0 = tc.y0;
        G.w = tc.w;
        G.h = tc.h;
        G.out_off = im.out_base;
        G.pitch_px = p.info.width;
        G.fmt = (int16_t)im.fmt;
        G.bitdepth = (int16_t)p.info.bitdepth;
        G.rev = (int8_t)rev;
        G.mct = (int8_t)p.info.mct;
        G.ncomp = (int8_t)nc;
        G.checkout = (int8_t)((im.checkout >= 0 && im.checkout < nc) ? im.checkout : -1);
        G.tiles_x = (tc.w + 63) / 64;
        const uint32_t gi = (uint32_t)groups.size();
        groups.push_back(G);
        for (int ty = 0; ty < (tc.h + 63) / 64; ++ty)
          for (int tx = 0; tx < G.tiles_x; ++tx) otasks.push_back({gi, (uint16_t)tx, (uint16_t)ty});
      }
    }
  }
  // work queue order: longest coded length first (counting sort on the length in 16-byte
  // steps, capped at 64 KB: linear time; order within a step is irrelevant to the queue)
  size_t n_ord = 0;
  for (auto &q : ordq) {
    constexpr int NB = 4096;
    std::vector<uint32_t> cnt(NB + 1, 0), tmp(q.size());
    auto key = [&](uint32_t i) { return NB - 1 - (int)(std::min<uint32_t>(cbs[i].data_len, 65535u) >> 4); };
    for (uint32_t i : q) cnt[key(i) + 1]++;
    for (int b = 0; b < NB; ++b) cnt[b + 1] += cnt[b];
    for (uint32_t i : q) tmp[cnt[key(i)]++] = i;
    q.swap(tmp);
    n_ord += q.size();
  }
  std::vector<uint32_t> dtask_off(2 * maxL + 1, 0);
  std::vector<DwtTask> dtasks;
  for (int s = 0; s < maxL; ++s) {
    dtask_off[2 * s] = (uint32_t)dtasks.size();
    dtasks.insert(dtasks.end(), steps_rev[s].begin(), steps_rev[s].end());
    dtask_off[2 * s + 1] = (uint32_t)dtasks.size();
    dtasks.insert(dtasks.end(), steps_irr[s].begin(), steps_irr[s].end());
  }
  dtask_off[2 * maxL] = (uint32_t)dtasks.size();

  // ---- staging layout (pinned)
  size_t o_cbs = 0;
  size_t o_ord = align_up(o_cbs + cbs.size() * sizeof(j2k_cblk), 256);
  size_t o_seg = align_up(o_ord + n_ord * 4, 256);
  size_t o_lev = align_up(o_seg + seg.size() * 4, 256);
  size_t o_dtk = align_up(o_lev + levels.size() * sizeof(DwtLevel), 256);
  size_t o_grp = align_up(o_dtk + dtasks.size() * sizeof(DwtTask), 256);
  size_t o_otk = align_up(o_grp + groups.size() * sizeof(OutGroup), 256);
  size_t o_fgr = align_up(o_otk + otasks.size() * sizeof(OutTask), 256);
  size_t o_ftk = align_up(o_fgr + fgroups.size() * sizeof(FusedGroup), 256);
  size_t o_ctk = align_up(o_ftk + (ftasks[0].size() + ftasks[1].size()) * sizeof(OutTask), 256);
  size_t o_byt = align_up(o_ctk + (ctasks[0].size() + ctasks[1].size()) * sizeof(CoarseTask), 256);
  size_t total = align_up(o_byt + S.bytes + 16, 256);
  if (c->h_stage_cap < total) {
    // double at least: page-locking is slow; the outgrown area is kept until ctx_destroy
    const size_t nc = std::max(total, c->h_stage_cap * 2);
    if (c->h_stage) c->h_retired.push_back(c->h_stage);
    c->h_stage = nullptr;
    c->h_stage_cap = 0;
    if (cudaMallocHost(&c->h_stage, nc) != cudaSuccess) {
      cudaGetLastError();
      return J2K_ERR_NOMEM;
    }
    c->h_stage_cap = nc;
  }
  uint8_t *H = (uint8_t *)c->h_stage;
  std::memcpy(H + o_cbs, cbs.data(), cbs.size() * sizeof(j2k_cblk));
  {
    size_t off = o_ord;
    for (auto &q : ordq) {
      std::memcpy(H + off, q.data(), q.size() * 4);
      off += q.size() * 4;
    }
  }
  std::memcpy(H + o_seg, seg.data(), seg.size() * 4);
  std::memcpy(H + o_lev, levels.data(), levels.size() * sizeof(DwtLevel));
  std::memcpy(H + o_dtk, dtasks.data(), dtasks.size() * sizeof(DwtTask));
  std::memcpy(H + o_grp, groups.data(), groups.size() * sizeof(OutGroup));
  std::memcpy(H + o_otk, otasks.data(), otasks.size() * sizeof(OutTask));
  std::memcpy(H + o_fgr, fgroups.data(), fgroups.size() * sizeof(FusedGroup));
  std::memcpy(H + o_ftk, ftasks[0].data(), ftasks[0].size() * sizeof(OutTask));
  std::memcpy(H + o_ftk + ftasks[0].size() * sizeof(OutTask), ftasks[1].data(), ftasks[1].size() * sizeof(OutTask));
  std::memcpy(H + o_ctk, ctasks[0].data(), ctasks[0].size() * sizeof(CoarseTask));
  std::memcpy(H + o_ctk + ctasks[0].size() * sizeof(CoarseTask), ctasks[1].data(), ctasks[1].size() * sizeof(CoarseTask));
  {
    // coded bytes of every image, copied by a few threads when there are many
    std::vector<std::pair<size_t, const j2k::ByteBuffer *>> parts;
    size_t off = o_byt;
    for (auto &im : c->imgs) {
      parts.push_back({off, &im.plan->p.bytes});
      off += im.plan->p.bytes.size();
    }
    auto copy_range = [&](size_t lo, size_t hi) {
      for (size_t k = lo; k < hi; ++k)
        if (!parts[k].second->empty()) std::memcpy(H + parts[k].first, parts[k].second->data(), parts[k].second->size());
    };
    const size_t nt = S.bytes > (8u << 20) ? std::min<size_t>(8, parts.size()) : 1;
    if (nt <= 1) {
      copy_range(0, parts.size());
    } else {
      std::vector<std::thread> th;
      for (size_t t = 0; t < nt; ++t)
        th.emplace_back(copy_range, parts.size() * t / nt, parts.size() * (t + 1) / nt);
      for (auto &x : th) x.join();
    }
  }

  // ---- device buffers
  int rc;
  if ((rc = ensure(c, c->d_cblks, o_byt)) != J2K_OK) return rc;  // all tables in one block
  if ((rc = ensure(c, c->d_bytes, S.bytes + 16)) != J2K_OK) return rc;
  if ((rc = ensure(c, c->d_status, S.cblks * 2 + 16)) != J2K_OK) return rc;
  if ((rc = ensure(c, c->d_counter, 64)) != J2K_OK) return rc;
  if ((rc = ensure(c, c->d_A, S.coef * 4 + 16)) != J2K_OK) return rc;
  if ((rc = ensure(c, c->d_B, S.coef * 4 + 16)) != J2K_OK) return rc;
  if ((rc = ensure(c, c->d_C, S.coef * 4 + 16)) != J2K_OK) return rc;
  if ((rc = ensure(c, c->d_out, S.out + 16)) != J2K_OK) return rc;
  uint8_t *D = (uint8_t *)c->d_cblks.p;
  c->launches = 0;

  CK(cudaEventRecord(c->ev[0], st));
  CK(cudaMemcpyAsync(D, H, o_byt, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(c->d_bytes.p, H + o_byt, S.bytes, cudaMemcpyHostToDevice, st));
  CK(cudaEventRecord(c->ev[1], st));
  for (int q = 0; q < NQ; ++q) c->sg.nq[q] = ordq[q].size();
  c->sg.n_cblks = S.cblks;
  c->sg.n_otasks = otasks.size();
  c->sg.o_fgr = o_fgr;
  c->sg.o_ftk = o_ftk;
  c->sg.n_ftasks[0] = ftasks[0].size();
  c->sg.n_ftasks[1] = ftasks[1].size();
  c->sg.o_ctk = o_ctk;
  c->sg.n_ctasks[0] = ctasks[0].size();
  c->sg.n_ctasks[1] = ctasks[1].size();
  c->sg.fwin = fwin;
  c->sg.o_cbs = o_cbs;
  c->sg.o_ord = o_ord;
  c->sg.o_seg = o_seg;
  c->sg.o_lev = o_lev;
  c->sg.o_dtk = o_dtk;
  c->sg.o_grp = o_grp;
  c->sg.o_otk = o_otk;
  c->sg.maxL = maxL;
  c->sg.dtask_off = dtask_off;
  if (c->h_status_cap < S.cblks + 1) {
    const size_t nc = std::max(S.cblks + 1, c->h_status_cap * 2);
    if (c->h_status) c->h_retired.push_back(c->h_status);
    c->h_status = nullptr;
    c->h_status_cap = 0;
    if (cudaMallocHost(&c->h_status, nc * 2) != cudaSuccess) {
      cudaGetLastError();
      return J2K_ERR_NOMEM;
    }
    c->h_status_cap = nc;
  }
  drop_graph(c);  // a captured decode belongs to the previous batch
  c->staged = true;
  c->launched = false;
  c->synced = false;
  return J2K_OK;
}

namespace {
// Event record that also fires when captured into a graph and replayed
cudaError_t record(cudaEvent_t ev, cudaStream_t st, bool capturing) {
  return capturing ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal) : cudaEventRecord(ev, st);
}

// Everything one decode of the staged batch enqueues after its input copies: counter reset,
// the Tier-1 launch, the DWT level launches, the output stage, the status read-back and the
// bracketing events.
int enqueue_decode(j2k_gpu_ctx *c, cudaStream_t st, bool capturing) {
  const auto &G = c->sg;
  uint8_t *D = (uint8_t *)c->d_cblks.p;
  const size_t o_cbs = G.o_cbs, o_ord = G.o_ord, o_seg = G.o_seg, o_lev = G.o_lev, o_dtk = G.o_dtk, o_grp = G.o_grp,
               o_otk = G.o_otk;
  const int maxL = G.maxL;
  const std::vector<uint32_t> &dtask_off = G.dtask_off;
  struct {
    size_t n;
    size_t size() const { return n; }
    bool empty() const { return n == 0; }
  } otasks{G.n_otasks};
  c->launches = 0;
  CK(cudaMemsetAsync(c->d_counter.p, 0, 64, st));

  // ---- Tier-1
  const j2k_cblk *d_cbs = (const j2k_cblk *)(D + o_cbs);
  const uint32_t *d_ord = (const uint32_t *)(D + o_ord);
  const uint32_t *d_seg = (const uint32_t *)(D + o_seg);
  int *cnt = (int *)c->d_counter.p;
  const auto *ltab = (const j2k_lanes::LaneTables *)c->d_tables.p;
  c->launches += launch_t1(c, st, G.nq, d_cbs, d_ord, cnt, d_seg, ltab);
  CK(cudaGetLastError());
  CK(record(c->ev[2], st, capturing));

  // ---- inverse DWT, coarsest level step first
  const DwtLevel *d_lev = (const DwtLevel *)(D + o_lev);
  const DwtTask *d_dtk = (const DwtTask *)(D + o_dtk);
  const float llg = j2k::irrev_ll_gain();
  const int dwt_cap = c->sm_count * 32;  // grid-stride cap: about three waves of resident CTAs
  for (int k = 0; k < 2; ++k) {
    const int n = (int)G.n_ctasks[k];
    if (!n) continue;
    const CoarseTask *ct = (const CoarseTask *)(D + G.o_ctk) + (k ? G.n_ctasks[0] : 0);
    if (k) dwt_coarse_kernel<true><<<std::min(n, dwt_cap), 128, 0, st>>>(ct, n, c->d_A.p, c->d_B.p, c->d_C.p, llg);
    else dwt_coarse_kernel<false><<<std::min(n, dwt_cap), 128, 0, st>>>(ct, n, c->d_A.p, c->d_B.p, c->d_C.p, llg);
    c->launches++;
  }
  for (int s = 0; s < maxL; ++s) {
    int n_rev = (int)(dtask_off[2 * s + 1] - dtask_off[2 * s]);
    int n_irr = (int)(dtask_off[2 * s + 2] - dtask_off[2 * s + 1]);
    if (n_rev) {
      dwt_level_kernel<true><<<std::min(n_rev, dwt_cap), DWT_THREADS, 0, st>>>(d_lev, d_dtk + dtask_off[2 * s], n_rev, c->d_A.p,
                                                                        c->d_B.p, c->d_C.p, llg);
      c->launches++;
    }
    if (n_irr) {
      dwt_level_kernel<false><<<std::min(n_irr, dwt_cap), DWT_THREADS, 0, st>>>(d_lev, d_dtk + dtask_off[2 * s + 1], n_irr,
                                                                         c->d_A.p, c->d_B.p, c->d_C.p, llg);
      c->launches++;
    }
  }
  for (int k = 0; k < 2; ++k) {
    const int nf = (int)G.n_ftasks[k];
    if (!nf) continue;
    const OutTask *ft = (const OutTask *)(D + G.o_ftk) + (k ? G.n_ftasks[0] : 0);
    const FusedGroup *fg = (const FusedGroup *)(D + G.o_fgr);
    if (k) {
      last_level_output_kernel<true><<<std::min(nf, dwt_cap), FUSED_THREADS, G.fwin * sizeof(DwtSmem<true>), st>>>(
          fg, ft, nf, c->d_A.p, c->d_B.p, c->d_C.p, llg, (uint8_t *)c->d_out.p);
    } else {
      last_level_output_kernel<false><<<std::min(nf, dwt_cap), FUSED_THREADS, G.fwin * sizeof(DwtSmem<false>), st>>>(
          fg, ft, nf, c->d_A.p, c->d_B.p, c->d_C.p, llg, (uint8_t *)c->d_out.p);
    }
    c->launches++;
  }
  if (!otasks.empty()) {
    output_kernel<<<std::min((int)otasks.size(), dwt_cap), 256, 0, st>>>(
        (const OutGroup *)(D + o_grp), (const OutTask *)(D + o_otk), (int)otasks.size(), c->d_A.p, c->d_B.p, c->d_C.p,
        (uint8_t *)c->d_out.p);
    c->launches++;
  }
  CK(cudaGetLastError());
  CK(record(c->ev[3], st, capturing));
  if (G.n_cblks) CK(cudaMemcpyAsync(c->h_status, c->d_status.p, G.n_cblks * 2, cudaMemcpyDeviceToHost, st));
  CK(record(c->ev[4], st, capturing));
  return J2K_OK;
}

// Capture the decode of the staged batch into a graph (once per staged batch).  Returns
// false when capture is unavailable, in which case the caller enqueues the launches
// directly; either way the same kernels run.
bool capture_decode(j2k_gpu_ctx *c, cudaStream_t st) {
  if (c->gexec) return true;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const int rc = enqueue_decode(c, st, true);
  const cudaError_t e = cudaStreamEndCapture(st, &g);
  if (rc != J2K_OK || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return false;
  }
  const cudaError_t ei = cudaGraphInstantiate(&c->gexec, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    c->gexec = nullptr;
    cudaGetLastError();
    return false;
  }
  c->graph_launches = c->launches;
  return true;
}

// Order of decodes on one device, across contexts.  Every run records `last` after its
// decode; a run whose Tier-1 launch fills every SM waits for it first.  The persistent
// Tier-1 kernel holds its SMs until its queue drains, so if it started while an earlier
// batch (of any context) was still in its Tier-1 tail, that batch's DWT levels could not
// run until this whole Tier-1 had finished.  Smaller Tier-1 launches leave SMs free and
// overlap the previous decode instead, which fills the idle SMs of latency-bound batches.
struct DeviceOrder {
  std::mutex mu;
  cudaEvent_t last = nullptr;
};
DeviceOrder &device_order(int device) {
  static DeviceOrder orders[64];
  return orders[device & 63];
}
}  // namespace

extern "C" int j2k_gpu_batch_run(j2k_gpu_ctx *c, void *user_stream) {
  if (!c) return J2K_ERR_ARG;
  if (!c->staged || (c->launched && !c->synced)) return J2K_ERR_STATE;
  cudaSetDevice(c->device);
  cudaStream_t st = user_stream ? (cudaStream_t)user_stream : c->stream;
  c->user_stream = st;
  // a stream the caller is capturing into a graph of its own gets no cross-capture
  // dependency: the caller's graph orders its work
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(st, &cap));
  const bool ordered = cap == cudaStreamCaptureStatusNone;
  DeviceOrder &order = device_order(c->device);
  std::lock_guard<std::mutex> lk(order.mu);
  if (!order.last) CK(cudaEventCreateWithFlags(&order.last, cudaEventDisableTiming));
  int t1_form = 0, t1_warps = 0;
  t1_shape(c, (int)c->sg.n_cblks, t1_form, t1_warps);
  const bool fills = (long long)c->sg.n_cblks >= (long long)c->sm_count * 32 ||
                     (t1_form == 3 && (long long)c->sg.nq[QL] >= c->sm_count);  // a lane-form CTA holds its SM
  if (ordered && fills) CK(cudaStreamWaitEvent(st, order.last, 0));
  if (c->launched) {
    // a repeated run: no input copies, both copy events at the start
    CK(cudaEventRecord(c->ev[0], st));
    CK(cudaEventRecord(c->ev[1], st));
  }  // else the first run after staging: the staging events already bracket the copies
  if (c->tuning.use_graph && capture_decode(c, st)) {
    CK(cudaGraphLaunch(c->gexec, st));
    c->launches = c->graph_launches;
  } else {
    const int rc = enqueue_decode(c, st, false);
    if (rc != J2K_OK) return rc;
  }
  if (ordered) CK(cudaEventRecord(order.last, st));
  c->launched = true;
  c->synced = false;
  c->copies_pending = false;
  return J2K_OK;
}

extern "C" int j2k_gpu_batch_launch(j2k_gpu_ctx *c, void *user_stream) {
  int rc = j2k_gpu_batch_stage(c, user_stream);
  if (rc != J2K_OK) return rc;
  return j2k_gpu_batch_run(c, user_stream);
}

extern "C" int j2k_gpu_batch_sync(j2k_gpu_ctx *c, int timeout_ms) {
  if (!c) return J2K_ERR_ARG;
  if (!c->launched) return J2K_ERR_STATE;
  if (c->synced) return J2K_OK;
  cudaSetDevice(c->device);
  auto t0 = std::chrono::steady_clock::now();
  // ev[5] is recorded after ev[4] on the same stream: it covers the decode and the copies
  cudaEvent_t done = c->copies_pending ? c->ev[5] : c->ev[4];
  for (;;) {
    cudaError_t e = cudaEventQuery(done);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return J2K_ERR_CUDA;
    if (timeout_ms == 0) return J2K_ERR_TIMEOUT;  // poll once
    if (timeout_ms >= 0) {
      auto el = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
      if (el > timeout_ms) return J2K_ERR_TIMEOUT;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  cudaEventElapsedTime(&c->t_h2d, c->ev[0], c->ev[1]);
  cudaEventElapsedTime(&c->t_t1, c->ev[1], c->ev[2]);
  cudaEventElapsedTime(&c->t_dwt, c->ev[2], c->ev[3]);
  cudaEventElapsedTime(&c->t_total, c->ev[0], c->ev[4]);
  for (auto &im : c->imgs) {
    int bad = 0;
    const size_t n = im.plan->p.cblks.size();
    for (size_t i = 0; i < n; ++i)
      if (c->h_status[im.cblk_base + i]) bad++;
    im.bad = bad;
    im.status = bad ? J2K_ERR_DECODE : J2K_OK;
  }
  c->synced = true;
  c->copies_pending = false;
  return J2K_OK;
}

extern "C" int j2k_gpu_image_status(const j2k_gpu_ctx *c, int slot, int *bad) {
  if (!c || slot < 0 || slot >= (int)c->imgs.size()) return J2K_ERR_ARG;
  if (!c->synced) return J2K_ERR_STATE;
  if (bad) *bad = c->imgs[slot].bad;
  return c->imgs[slot].status;
}

extern "C" int j2k_gpu_output_device(const j2k_gpu_ctx *c, int slot, const void **dptr, size_t *bytes) {
  if (!c || slot < 0 || slot >= (int)c->imgs.size() || !dptr) return J2K_ERR_ARG;
  if (!c->launched) return J2K_ERR_STATE;
  *dptr = (const uint8_t *)c->d_out.p + c->imgs[slot].out_base;
  if (bytes) *bytes = c->imgs[slot].out_bytes;
  return J2K_OK;
}

extern "C" int j2k_gpu_output_copy(j2k_gpu_ctx *c, int slot, void *dst, size_t bytes) {
  if (!c || slot < 0 || slot >= (int)c->imgs.size() || !dst) return J2K_ERR_ARG;
  if (!c->synced) return J2K_ERR_STATE;
  const BatchImage &im = c->imgs[slot];
  if (bytes < im.out_bytes) return J2K_ERR_ARG;
  cudaSetDevice(c->device);
  CK(cudaMemcpyAsync(dst, (const uint8_t *)c->d_out.p + im.out_base, im.out_bytes, cudaMemcpyDeviceToHost,
                     c->user_stream));
  CK(cudaStreamSynchronize(c->user_stream));
  return J2K_OK;
}

extern "C" int j2k_gpu_output_copy_async(j2k_gpu_ctx *c, int slot, void *dst, size_t bytes) {
  if (!c || slot < 0 || slot >= (int)c->imgs.size() || !dst) return J2K_ERR_ARG;
  if (!c->launched || c->synced) return J2K_ERR_STATE;
  const BatchImage &im = c->imgs[slot];
  if (bytes < im.out_bytes) return J2K_ERR_ARG;
  cudaSetDevice(c->device);
  CK(cudaMemcpyAsync(dst, (const uint8_t *)c->d_out.p + im.out_base, im.out_bytes, cudaMemcpyDeviceToHost,
                     c->user_stream));
  CK(cudaEventRecord(c->ev[5], c->user_stream));
  c->copies_pending = true;
  return J2K_OK;
}

namespace {
// copy a tile-component region of buffer `buf` to the host
int copy_region(j2k_gpu_ctx *c, const void *buf, uint64_t off, size_t elems, void *dst) {
  CK(cudaMemcpyAsync(dst, (const uint8_t *)buf + off * 4, elems * 4, cudaMemcpyDeviceToHost, c->user_stream));
  return J2K_OK;
}
}  // namespace

extern "C" int j2k_gpu_coefficients_copy(j2k_gpu_ctx *c, int slot, int stage, void *dst, size_t bytes) {
  if (!c || slot < 0 || slot >= (int)c->imgs.size() || !dst) return J2K_ERR_ARG;
  if (!c->synced) return J2K_ERR_STATE;
  const BatchImage &im = c->imgs[slot];
  const auto &p = im.plan->p;
  if (bytes < p.info.coef_elems * 4) return J2K_ERR_ARG;
  if (stage == 1 && im.fused) return J2K_ERR_STATE;  // last level fused with the output stage
  cudaSetDevice(c->device);
  for (const j2k_tilecomp &tc : p.tilecomps) {
    const int Lt = tc.levels;
    const void *buf = c->d_A.p;
    if (stage == 1 && Lt > 0) buf = (Lt & 1) ? c->d_B.p : c->d_C.p;
    int rc = copy_region(c, buf, im.coef_base + tc.coef_off, (size_t)tc.w * tc.h, (uint8_t *)dst + tc.coef_off * 4);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(c->user_stream));
  return J2K_OK;
}

extern "C" int j2k_gpu_component_copy(j2k_gpu_ctx *c, int slot, int comp, void *dst, size_t bytes) {
  if (!c || slot < 0 || slot >= (int)c->imgs.size() || !dst) return J2K_ERR_ARG;
  if (!c->synced) return J2K_ERR_STATE;
  const BatchImage &im = c->imgs[slot];
  const auto &p = im.plan->p;
  if (comp < 0 || comp >= p.info.ncomp) return J2K_ERR_ARG;
  // the component on its own grid (smaller than the picture when sub-sampled)
  const int cw = p.info.comp_w[comp], ch = p.info.comp_h[comp];
  const size_t need = (size_t)cw * ch * 4;
  if (bytes < need) return J2K_ERR_ARG;
  if (im.fused) return J2K_ERR_STATE;  // last level fused with the output stage
  cudaSetDevice(c->device);
  bool found = false;
  for (const j2k_tilecomp &tc : p.tilecomps) {
    if (tc.comp != comp) continue;
    found = true;
    const int Lt = tc.levels;
    const void *buf = Lt == 0 ? c->d_A.p : ((Lt & 1) ? c->d_B.p : c->d_C.p);
    CK(cudaMemcpy2DAsync((uint8_t *)dst + ((size_t)tc.y0 * cw + tc.x0) * 4, (size_t)cw * 4,
                         (const uint8_t *)buf + (im.coef_base + tc.coef_off) * 4, (size_t)tc.w * 4, (size_t)tc.w * 4,
                         tc.h, cudaMemcpyDeviceToHost, c->user_stream));
  }
  if (!found) return J2K_ERR_ARG;
  CK(cudaStreamSynchronize(c->user_stream));
  return J2K_OK;
}

extern "C" int j2k_gpu_last_timing(const j2k_gpu_ctx *c, float *t1, float *dwt, float *h2d, float *total) {
  if (!c || !c->synced) return J2K_ERR_STATE;
  if (t1) *t1 = c->t_t1;
  if (dwt) *dwt = c->t_dwt;
  if (h2d) *h2d = c->t_h2d;
  if (total) *total = c->t_total;
  return J2K_OK;
}

extern "C" int j2k_gpu_autotune(j2k_gpu_ctx *c, void *stream, int iters, j2k_gpu_tuning *best, float *best_ms) {
  if (!c || iters <= 0) return J2K_ERR_ARG;
  if (!c->staged || (c->launched && !c->synced)) return J2K_ERR_STATE;
  const j2k_gpu_tuning saved = c->tuning;
  const int n = (int)(c->sg.nq[QL] + c->sg.nq[QW]);
  const int bucket = n > 0 ? 31 - __builtin_clz((unsigned)n) : 0;
  j2k_gpu_ctx::TuneEntry win;
  win.t1_ms = 1e30f;
  static const int forms[2] = {1, 2};
  static const int widths[3] = {2, 4, 8};
  for (int f : forms)
    for (int w : widths) {
      j2k_gpu_tuning t = saved;
      t.t1_form = f;
      t.t1_warps_per_cta = w;
      t.use_graph = 0;
      int rc = j2k_gpu_set_tuning(c, &t);
      float tmin = 1e30f;
      for (int i = 0; rc == J2K_OK && i <= iters; ++i) {
        if ((rc = j2k_gpu_batch_run(c, stream)) != J2K_OK || (rc = j2k_gpu_batch_sync(c, -1)) != J2K_OK) break;
        if (i > 0) tmin = std::min(tmin, c->t_t1);  // the first run warms caches and clocks
      }
      if (rc != J2K_OK) {
        c->tuning = saved;
        return rc;
      }
      if (tmin < win.t1_ms) {
        win.t1_ms = tmin;
        win.form = f;
        win.warps = w;
      }
    }
  c->tune_table[bucket] = win;
  // DWT: the coarse levels in one shared-memory kernel, or one launch per level.  The choice
  // shapes the staged task tables, so each candidate re-stages the batch; the winner is kept
  // for the auto setting (dwt_coarse 0) and the batch is staged again with the caller's
  // tuning at the end.
  int dwt_win = 1;
  float dwt_best = 1e30f;
  for (int cand : {1, 2}) {
    j2k_gpu_tuning t = saved;
    t.t1_form = win.form;
    t.t1_warps_per_cta = win.warps;
    t.use_graph = 0;
    t.dwt_coarse = cand;
    int rc = j2k_gpu_set_tuning(c, &t);
    if (rc == J2K_OK) rc = j2k_gpu_batch_stage(c, stream);
    float tmin = 1e30f;
    for (int i = 0; rc == J2K_OK && i <= iters; ++i) {
      if ((rc = j2k_gpu_batch_run(c, stream)) != J2K_OK || (rc = j2k_gpu_batch_sync(c, -1)) != J2K_OK) break;
      if (i > 0) tmin = std::min(tmin, c->t_dwt);
    }
    if (rc != J2K_OK) {
      c->tuning = saved;
      return rc;
    }
    if (tmin < dwt_best) {
      dwt_best = tmin;
      dwt_win = cand;
    }
  }
  c->dwt_auto = dwt_win;
  c->tuning = saved;
  const int rs = j2k_gpu_batch_stage(c, stream);
  if (rs != J2K_OK) return rs;
  drop_graph(c);
  if (best) {
    *best = saved;
    best->t1_form = win.form;
    best->t1_warps_per_cta = win.warps;
    best->dwt_coarse = dwt_win;
  }
  if (best_ms) *best_ms = win.t1_ms;
  return J2K_OK;
}

extern "C" int j2k_gpu_last_launches(const j2k_gpu_ctx *c, int *n) {
  if (!c || !n) return J2K_ERR_ARG;
  *n = c->launches;
  return J2K_OK;
}

extern "C" int j2k_gpu_decode(j2k_gpu_ctx *c, const uint8_t *cs, size_t len, int fmt, int flags, void *host_out,
                              size_t host_out_bytes) {
  if (!c || !cs || !host_out) return J2K_ERR_ARG;
  j2k_plan *p = nullptr;
  int rc = j2k_plan_create(cs, len, 0, 0, 0, &p);
  if (rc) return rc;
  if ((rc = j2k_gpu_batch_begin(c)) == J2K_OK && (rc = j2k_gpu_batch_add(c, p, fmt, flags, nullptr)) == J2K_OK &&
      (rc = j2k_gpu_batch_launch(c, nullptr)) == J2K_OK && (rc = j2k_gpu_batch_sync(c, -1)) == J2K_OK) {
    rc = j2k_gpu_output_copy(c, 0, host_out, host_out_bytes);
    if (rc == J2K_OK) rc = j2k_gpu_image_status(c, 0, nullptr);
  }
  j2k_gpu_batch_begin(c);
  j2k_plan_destroy(p);
  return rc;
}

int bmi_engine::set_checkout(j2k_gpu_ctx *c, int slot, int comp) {
  if (!c || slot < 0 || slot >= (int)c->imgs.size()) return J2K_ERR_ARG;
  if (c->launched) return J2K_ERR_STATE;
  c->imgs[slot].checkout = comp;
  return J2K_OK;
}
