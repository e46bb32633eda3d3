/*
 * ref_cpu_driver.cpp — C entry points into the reference's own CPU decoder (BMI::Decoder,
 * decoder/common/include/codec_base.h:316-345; engine decoder/core/src/decoderconcrete.cpp),
 * compiled from the reference tree by oracle/build_ref_cpu.sh into oracle/_ref/libref_cpu.so.
 * TEST AND BASELINE INFRASTRUCTURE ONLY: tests/ pin the oracle and the device path to its
 * output, and bench.py's CPU arm times it.  Nothing in the product links it.
 *
 * The engine is the reference's singleton: ref_cpu_init configures it once per process
 * (EnginConfig with mUsingGpu = false, since the reference's CUDA-1.0 back end does not
 * build; mThreadNum given explicitly because its Linux Init otherwise runs one worker,
 * decoderconcrete.cpp:136-153).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <new>

#include "codec_base.h"

/* Zero-filled heap for the reference's objects.  Its job queue leaves a member
 * uninitialised outside Windows (SemaphoreControledJobQueue::mInited, initialised only under
 * `#if _WINDOWS` in decoder/core/include/jobqueue.h), and Init (jobqueue.cpp:15-26) then
 * skips creating its semaphore and mutex whenever the heap hands back non-zero memory: the
 * engine hangs or aborts in pthread_mutex_lock at random.  Allocating zeroed memory, as a
 * fresh heap gives, removes that without touching the reference's code.  The library is
 * linked with -Bsymbolic so these replace operator new only inside it. */
void *operator new(size_t n) throw(std::bad_alloc) {
  void *p = calloc(1, n ? n : 1);
  if (!p) throw std::bad_alloc();
  return p;
}
void *operator new[](size_t n) throw(std::bad_alloc) { return operator new(n); }
void operator delete(void *p) throw() { free(p); }
void operator delete[](void *p) throw() { free(p); }

namespace {
bool g_inited = false;
double now_ms() {
  timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec * 1e3 + t.tv_nsec * 1e-6;
}
}  // namespace

/* Start the engine with `threads` worker threads; returns the count the engine runs. */
extern "C" int ref_cpu_init(int threads) {
  if (g_inited) return BMI::Decoder::Get()->GetEngineConfig()->mThreadNum;
  BMI::EnginConfig cfg;
  cfg.mUsingGpu = false;
  cfg.mSyncMode = true;
  cfg.mThreadNum = threads > 0 ? threads : 1;
  cfg.mInputQueueLen = 1;
  cfg.mOutputQueueLen = 1;
  int n = BMI::Decoder::Get()->Init(&cfg);
  g_inited = true;
  return n;
}

/* Decode one codestream into `out` (packed in the reference's OutputFormat `out_format`)
 * with `top_level` as DecodeJobConfig::mDwtDecodeTopLevel (-1 = full resolution).
 * Returns the BMI::Status of the decode (0 = READY); on READY, `out_bytes` receives the
 * result size (copied when it fits `cap`), `w`/`h` the output size and `ms` the wall time of
 * Decode() + GetResult(). */
extern "C" int ref_cpu_decode(const uint8_t *cs, int len, int out_format, int top_level, uint8_t *out, long cap,
                              int *w, int *h, int *out_bytes, double *ms) {
  if (!g_inited) ref_cpu_init(1);
  BMI::Decoder *dec = BMI::Decoder::Get();
  BMI::DecodeJobConfig jc;
  jc.mOutputFormat = (OutputFormat)out_format;
  jc.mDwtDecodeTopLevel = top_level;
  dec->SetJobConfig(jc);
  double t0 = now_ms();
  BMI::CodeStreamHandler hd = dec->Decode(cs, len);
  BMI::Status st = dec->CheckStatus(hd);
  int size = 0;
  const void *res = NULL;
  if (st == BMI::READY) res = dec->GetResult(hd, size);
  double t1 = now_ms();
  if (ms) *ms = t1 - t0;
  if (st != BMI::READY) return (int)st;
  BMI::CodeStreamProperties p;
  memset(&p, 0, sizeof(p));
  if (dec->CheckProperties(hd, p)) {
    if (w) *w = p.mOutputSize.x;
    if (h) *h = p.mOutputSize.y;
  }
  if (out_bytes) *out_bytes = size;
  if (res && out && size <= cap) memcpy(out, res, (size_t)size);
  dec->Release(hd);
  return res ? 0 : -1;
}
