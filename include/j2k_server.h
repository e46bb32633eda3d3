/*
 * j2k_server.h — continuous-batching decode service on one GPU.
 *
 * Callers submit codestreams as they arrive and wait for (or poll) each result.  A
 * scheduler thread merges whatever is pending into the next batch as soon as a pipeline
 * slot and device memory allow (one shared Tier-1 launch and shared DWT level launches per
 * batch), so requests that arrive while earlier batches run on the GPU are admitted into
 * the next slot and their work overlaps on the device.  Each slot keeps its device buffers
 * (coded bytes, coefficients, outputs) and pinned output staging between batches.
 *
 * Counterpart in the reference: the asynchronous BMI::Decoder queue
 * (decoder/common/include/codec_base.h:190-200 mOutputQueueLen, :320-341 Decode /
 * CheckStatus / GetResult / Release) and the batchdecode driver loop
 * (batchdecode/batchdecode.cpp), which decode one picture per engine job.
 *
 * Thread safety: submit / wait / poll / release / stats may be called from any threads.
 */
#ifndef J2K_SERVER_H
#define J2K_SERVER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct j2k_server j2k_server;

typedef struct j2k_server_config {
  int device;
  size_t mem_budget;    /* device bytes for all pipeline slots together (0 = 60% of free) */
  int pipeline_depth;   /* batches in flight at once (0 = 2) */
  int max_batch_images; /* images per batch (0 = no limit besides memory) */
  uint64_t max_batch_pixels; /* pixels per batch (0 = 128 M): bounds the host staging of one
                                batch so that it overlaps the device work of the previous one */
} j2k_server_config;

typedef struct j2k_server_stats {
  uint64_t completed, failed, batches;
  double mean_batch_images;
  double p50_us, p99_us, max_us;  /* submit -> result on the host, over completed requests */
  double busy_s;                   /* wall time with at least one batch in flight */
  uint64_t pixels;                 /* decoded pixels of completed requests */
  uint64_t launches;               /* kernel launches enqueued by all batches */
  double gpu_ms;                   /* device time of all batches (first to last event) */
  double stage_ms;                 /* host time spent assembling and enqueueing batches */
  double enqueue_ms;               /* ... of which in j2k_gpu_batch_launch */
  uint64_t pool_growths;           /* batches that had to enlarge a slot's device pool */
  uint64_t pinned_allocs;          /* page-locked chunks added to the output arena (>= 256 MB each) */
} j2k_server_stats;

/* Starts the scheduler thread.  J2K_ERR_NODEVICE without a CUDA device. */
int j2k_server_create(const j2k_server_config *cfg, j2k_server **out);
/* Finishes the batches in flight, fails the requests still pending, joins the thread. */
void j2k_server_destroy(j2k_server *srv);

/* Copies the codestream, runs Tier-2 on the calling thread and queues the request.
 * Returns a request id >= 0, or a negative j2k_status (J2K_ERR_PARSE, J2K_ERR_NOMEM when the
 * picture alone exceeds one slot's share of the budget). */
int64_t j2k_server_submit(j2k_server *srv, const void *codestream, size_t len, int out_format, int flags);

/* Waits for a request (timeout_ms < 0 = forever, 0 = poll).  Returns J2K_OK / the decode
 * status, J2K_ERR_TIMEOUT while it is still queued or running.  When `dst` is not NULL the
 * packed output is copied there (`cap` bytes available); `bytes` receives its size. */
int j2k_server_wait(j2k_server *srv, int64_t id, void *dst, size_t cap, size_t *bytes, int timeout_ms);
/* Like wait, without a copy: `*ptr` points at the packed output in the server's pinned host
 * memory, valid until j2k_server_release (the reference's GetResult / Release contract). */
int j2k_server_result(j2k_server *srv, int64_t id, const void **ptr, size_t *bytes, int timeout_ms);
/* Submit-to-completion latency of a finished request, in microseconds. */
int j2k_server_latency_us(j2k_server *srv, int64_t id, double *us);
/* Drops a finished request and its output (not concurrently with a wait() on the same id). */
int j2k_server_release(j2k_server *srv, int64_t id);
/* Blocks until every submitted request has finished. */
int j2k_server_drain(j2k_server *srv);
int j2k_server_stats_get(j2k_server *srv, j2k_server_stats *st);
/* Clears the latency / batch statistics (requests are not affected). */
int j2k_server_stats_reset(j2k_server *srv);

#ifdef __cplusplus
}
#endif
#endif
