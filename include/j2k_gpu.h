/*
 * j2k_gpu.h — thin C ABI between the host JPEG 2000 front end and the sm_100a decode path.
 *
 * Plain pointers and sizes only; no exceptions cross this boundary; every call returns a
 * j2k_status (0 = ok, negative = error).  Thread safety: one submitting thread and one
 * completion thread per context.
 *
 * This ABI replaces the reference's internal GPU boundary:
 *   - CudaManager (decoder/cudainterface/include/cudaInterface.h, cudainterface.cpp:316-2800):
 *     Init / InitPicture / GetStripeBuffer / UploadStripeBuf / GetResultBuf / GetOneComponent
 *     / ReleaseCudaJob / ThreadSafeWaitForCudaThreadFinish;
 *   - the gpulib C ABI (decoder/cudainterface/include/gpulib.h:24-57): GpuInit,
 *     MallocGpuBuf, Gpu2DCopy, BMI_comp_idwt, BMI_resolution_idwt, BMI_tile_MCT /
 *     BMI_tile_ICT / BMI_tile_Merge, BMI_tile_One_Component, BMI_Comp_DC_SHIFT.
 * Unlike the reference (host Tier-1 on worker threads, then per-stripe H2D copies), the
 * whole Tier-1 + dequantisation + inverse DWT + inverse MCT runs on the device from the
 * coded bytes the host Tier-2 collected.
 */
#ifndef J2K_GPU_H
#define J2K_GPU_H

#include <stddef.h>
#include <stdint.h>

#include "../jpeg2000-decoder_b200/csrc/plan.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum j2k_status {
  J2K_OK = 0,
  J2K_ERR_ARG = -1,
  J2K_ERR_PARSE = -2,
  J2K_ERR_UNSUPPORTED = -3,
  J2K_ERR_CUDA = -4,
  J2K_ERR_NOMEM = -5,     /* device-memory budget exceeded */
  J2K_ERR_TIMEOUT = -6,
  J2K_ERR_DECODE = -7,    /* at least one code-block reported a Tier-1 error */
  J2K_ERR_STATE = -8,
  J2K_ERR_NODEVICE = -9
} j2k_status;

/* OutputFormat of the reference (decoder/common/include/codec_datatype.h:38-51) */
enum {
  J2K_FMT_32BITS_ARGB = 0,
  J2K_FMT_48BITS_RGB = 1,
  J2K_FMT_24BITS_RGB = 2,
  J2K_FMT_32BITS_4COMPONENTS = 3,
  J2K_FMT_64BITS_4COMPONENTS = 4,
  J2K_FMT_48BITS_3COMPONENTS = 5,
  J2K_FMT_24BITS_3COMPONENTS = 6,
  J2K_FMT_NONE = 7,             /* components only (GetDecodedComponentInt / Float) */
  J2K_FMT_64BITS_ARGB = 8
};

/* decode flags */
enum {
  J2K_FLAG_REF_COMPAT = 0x1, /* reproduce the reference's 5/3 column-end arithmetic
                                (bmi_cpu_dwt_decoder.cpp:3364-3398) instead of T.800 */
  J2K_FLAG_KEEP_COMPONENTS = 0x2 /* keep the reconstructed components in device memory for
                                    j2k_gpu_component_copy / coefficients_copy(stage 1).
                                    Without it an image with a packed output format has its
                                    last DWT level fused with the inverse MCT and pack, which
                                    never stores the components. */
};

/* ---------------------------------------------------------------- host plans (Tier-2) */
typedef struct j2k_plan j2k_plan;

/* Parse a J2K codestream (or JP2 file) and run Tier-2 on the host.  `discard_levels`
 * decodes at 1/2^n resolution (reference DecodeJobConfig::mDwtDecodeTopLevel);
 * `max_layers` 0 = all; bit c of `ignore_components` skips component c. */
int j2k_plan_create(const uint8_t *codestream, size_t len, int discard_levels, int max_layers,
                    unsigned ignore_components, j2k_plan **out);
/* The same with the Tier-2 of a multi-tile picture spread over `threads` host threads (tiles
 * are independent; the plan is identical for any thread count).  The counterpart of the
 * reference's worker-thread count (EnginConfig::mThreadNum, codec_base.h; BMI_dec_init's
 * thread_num, bmi_jp2dec.h:82) for the part of the decode that stays on the host. */
int j2k_plan_create_mt(const uint8_t *codestream, size_t len, int discard_levels, int max_layers,
                       unsigned ignore_components, int threads, j2k_plan **out);
void j2k_plan_destroy(j2k_plan *plan);
int j2k_plan_info(const j2k_plan *plan, j2k_image_info *info);
const j2k_cblk *j2k_plan_cblks(const j2k_plan *plan);
const uint32_t *j2k_plan_seglens(const j2k_plan *plan);
const uint8_t *j2k_plan_bytes(const j2k_plan *plan);
const j2k_tilecomp *j2k_plan_tilecomps(const j2k_plan *plan);
/* bytes of packed output for a format (0 for J2K_FMT_NONE) */
size_t j2k_output_bytes(const j2k_image_info *info, int format);
const char *j2k_status_string(int status);

/* ---------------------------------------------------------------- device context ---- */
typedef struct j2k_gpu_ctx j2k_gpu_ctx;

/* Create a context on `device`.  `mem_budget` bounds the device pool (0 = 80% of free
 * memory).  Fails with J2K_ERR_NODEVICE when no CUDA device is present: there is no CPU
 * fallback. */
int j2k_gpu_ctx_create(int device, size_t mem_budget, j2k_gpu_ctx **out);
void j2k_gpu_ctx_destroy(j2k_gpu_ctx *ctx);
/* Device pool bytes currently reserved / the budget. */
int j2k_gpu_mem_usage(const j2k_gpu_ctx *ctx, size_t *reserved, size_t *budget);

/* A batch collects images whose code-blocks share one Tier-1 launch and whose DWT levels
 * share the level launches.  Slots are numbered from 0 in add order. */
int j2k_gpu_batch_begin(j2k_gpu_ctx *ctx);
int j2k_gpu_batch_add(j2k_gpu_ctx *ctx, const j2k_plan *plan, int out_format, int flags, int *slot);
/* Device bytes the current batch needs (admission control against the budget). */
int j2k_gpu_batch_footprint(const j2k_gpu_ctx *ctx, size_t *bytes);
/* Stage inputs (pinned host -> device) and enqueue all kernels on `stream`
 * (a cudaStream_t, or NULL for the context's stream).  Asynchronous. */
int j2k_gpu_batch_launch(j2k_gpu_ctx *ctx, void *stream);
/* The two halves of batch_launch: stage assembles the batch's work lists and coded bytes
 * in pinned memory and copies them to the device; run enqueues Tier-1, the DWT levels and
 * the output stage on the staged (device-resident) inputs.  run may be repeated after a
 * sync to decode the same staged batch again. */
int j2k_gpu_batch_stage(j2k_gpu_ctx *ctx, void *stream);
int j2k_gpu_batch_run(j2k_gpu_ctx *ctx, void *stream);
/* Wait for the batch with a host-side timeout (ms, < 0 = forever, 0 = poll once and return
 * J2K_ERR_TIMEOUT while the batch is still running). */
int j2k_gpu_batch_sync(j2k_gpu_ctx *ctx, int timeout_ms);
/* Per-image status after sync: J2K_OK or J2K_ERR_DECODE; `bad_blocks` may be NULL. */
int j2k_gpu_image_status(const j2k_gpu_ctx *ctx, int slot, int *bad_blocks);
/* Packed output of a slot (device pointer valid until the next batch_begin). */
int j2k_gpu_output_device(const j2k_gpu_ctx *ctx, int slot, const void **dptr, size_t *bytes);
int j2k_gpu_output_copy(j2k_gpu_ctx *ctx, int slot, void *host_dst, size_t bytes);
/* Enqueue the copy of a slot's packed output into `host_dst` behind the batch's decode,
 * between batch_launch (or batch_run) and batch_sync.  The copy overlaps whatever the host
 * does next; batch_sync returns only once every copy enqueued this way has landed, so
 * `host_dst` (pinned memory, for the copy to be asynchronous) must stay valid until then.
 * The counterpart of a GetResult into the output queue without a host wait per picture. */
int j2k_gpu_output_copy_async(j2k_gpu_ctx *ctx, int slot, void *host_dst, size_t bytes);
/* Decoded (un-shifted) component samples of a slot as int32 (5/3) or float32 (9/7),
 * row-major over the output size: the reference's GetDecodedComponentInt / Float
 * (decoder/core/src/decoderconcrete.cpp:531-584).  J2K_ERR_STATE for an image added with a
 * packed format and without J2K_FLAG_KEEP_COMPONENTS. */
int j2k_gpu_component_copy(j2k_gpu_ctx *ctx, int slot, int comp, void *host_dst, size_t bytes);
/* Parity hooks: the coefficient buffer of a slot after Tier-1 (stage 0) or after the
 * inverse DWT of every tile-component (stage 1), in the plan's Mallat layout. */
int j2k_gpu_coefficients_copy(j2k_gpu_ctx *ctx, int slot, int stage, void *host_dst, size_t bytes);

/* Kernel-level timing of the last synced batch (ms, from CUDA events on the launch
 * stream): Tier-1, inverse DWT + MCT, H2D, D2H.  NULL pointers are skipped. */
int j2k_gpu_last_timing(const j2k_gpu_ctx *ctx, float *t1_ms, float *dwt_ms, float *h2d_ms, float *total_ms);
/* Number of kernel launches enqueued by the last batch_launch. */
int j2k_gpu_last_launches(const j2k_gpu_ctx *ctx, int *launches);

/* Tuning knobs picked by the autotuner (0 = default). */
typedef struct j2k_gpu_tuning {
  int t1_warps_per_cta;  /* code-blocks decoded concurrently per CTA */
  int dwt_tile;          /* output tile edge of the DWT level kernels (64; other values are refused) */
  int use_graph;         /* capture Tier-1 + DWT launches of a batch into a CUDA graph */
  int t1_form;           /* Tier-1 kernel form: 0 auto, 1 compact (one block per warp, throughput),
                            2 unrolled (one block per warp, latency), 3 lanes (one block per lane;
                            bypass blocks of the batch go to the compact form; slower than 1 on
                            the measured workloads, never chosen by the auto form; switching to or
                            from 3 takes effect at the next stage) */
  int t1_latency_waves;  /* auto form without an autotuned choice: unrolled while code-blocks <=
                            this many x 32 warps x SMs, compact above */
  int dwt_coarse;        /* the coarse levels of each tile-component (resolutions up to 64 samples a
                            side) in one shared-memory kernel: 0 default (on), 1 on, 2 off (one
                            launch per level) */
} j2k_gpu_tuning;
int j2k_gpu_set_tuning(j2k_gpu_ctx *ctx, const j2k_gpu_tuning *t);
int j2k_gpu_get_tuning(const j2k_gpu_ctx *ctx, j2k_gpu_tuning *t);
/* Autotuner: times the staged batch (`iters` runs after one warm-up run per candidate)
 * under the compact and unrolled Tier-1 kernel forms and CTA widths (2, 4, 8 warps) and
 * records the fastest for batches of this many code-blocks (power-of-two bucket); the
 * auto form (t1_form 0) then uses it for every later batch in that bucket.  Then, with that
 * Tier-1 shape, it times the inverse DWT with the coarse levels fused into one
 * shared-memory kernel and with one launch per level (re-staging the batch for each) and
 * keeps the faster for dwt_coarse 0.  The context's own tuning is left as it was and the
 * batch is staged again with it; `best` / `best_ms` (may be NULL) receive the winner and
 * its Tier-1 time.  The staged batch can be run again afterwards. */
int j2k_gpu_autotune(j2k_gpu_ctx *ctx, void *stream, int iters, j2k_gpu_tuning *best, float *best_ms);

/* Inverse DWT of one tile-component that allocates no device memory, for callers that
 * cannot call cudaMalloc (inside stream capture, in real-time callbacks, or under a host
 * that owns every device buffer).  No counterpart in the reference.  `coef`: device
 * pointer to the tile-component's Tier-1 coefficients in the plan's Mallat layout (row
 * stride tc->w; int32 for 5/3, float for 9/7, as j2k_gpu_coefficients_copy stage 0 lays
 * them out); `out`: device pointer receiving the reconstructed samples (row stride
 * `out_stride` elements, the values of j2k_gpu_component_copy).  Intermediate levels use a
 * static device array of J2K_NOALLOC_SCRATCH_BYTES held by every GPU that loads the
 * library; tile-components needing more than that (2 * res_w[L-1] * res_h[L-1] * 4 bytes)
 * return J2K_ERR_UNSUPPORTED.  The first call on a device looks up the array's device
 * address (make it before any stream capture); the address is kept for the life of the
 * process, so a caller that resets the device must restart the process before calling
 * again.  Overlapping calls race on the array.  A resolution table that does not nest
 * inside the tile-component returns J2K_ERR_ARG before anything is enqueued; a CUDA error
 * already pending from earlier work returns J2K_ERR_CUDA and stays pending.
 * Asynchronous on `stream`. */
#define J2K_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)
int j2k_gpu_tile_idwt_noalloc(const j2k_tilecomp *tc, int reversible, int flags, const void *coef, void *out,
                              int out_stride, void *stream);

/* One-call convenience: decode one codestream into host memory (pinned staging inside). */
int j2k_gpu_decode(j2k_gpu_ctx *ctx, const uint8_t *codestream, size_t len, int out_format, int flags,
                   void *host_out, size_t host_out_bytes);

#ifdef __cplusplus
}
#endif
#endif
