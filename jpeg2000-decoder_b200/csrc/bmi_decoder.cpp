/*
 * bmi_decoder.cpp — BMI::Decoder (include/bmi_decoder.h) on the GPU decode path.
 *
 * Mirrors the reference engine's public behaviour (decoder/core/src/decoderconcrete.cpp):
 * a singleton (decoder.cpp:77-92) with a ring of output slots of mOutputQueueLen entries;
 * Decode() returns a monotonically increasing handler (:318-320, :435); a slot
 * overwritten by a later decode reports RELEASED (:447-453); GetResult() returns the
 * packed picture in the job's OutputFormat; GetDecodedComponentInt/Float return the
 * un-shifted component samples (int for 5/3, float for 9/7, :531-584); PreDecode() parses
 * the main header only (:741-764).  In synchronous mode Decode() blocks until the picture
 * is ready (:771-774); in asynchronous mode it returns after the launch and CheckStatus()
 * reports DECODING until the device finishes.
 *
 * Differences: there is no worker-thread pool or CPU DWT; Tier-2 runs on the calling
 * thread and everything after it on the device.  mUsingGpu = false is rejected (no CPU
 * fallback) and Init() fails when no CUDA device is present.
 */
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/bmi_decoder.h"
#include "../../include/bmi_decoder_c.h"
#include "../../include/j2k_gpu.h"
#include "bmi_engine.h"
#include "codestream.h"

namespace {

using namespace BMI;

struct Slot {
  CodeStreamHandler handler = INVALID;
  Status status = INVALID_STATUS;
  DecodeJobConfig cfg;
  CodeStreamProperties props{};
  std::vector<uint8_t> codestream;
  std::vector<uint8_t> result, thumb;
  std::vector<int32_t> comp_int;
  std::vector<float> comp_float;
  int comp_loaded = -1;
  bool pending = false;
  int gpu_slot = -1;
  int comp_w[J2K_MAX_COMPONENTS] = {0}, comp_h[J2K_MAX_COMPONENTS] = {0};  // each component's own grid
};

int fmt_bytes(int fmt) {
  switch (fmt) {
    case IMAGE_FOTMAT_32BITS_ARGB:
    case IMAGE_FOTMAT_32BITS_4COMPONENTS: return 4;
    case IMAGE_FOTMAT_48BITS_RGB:
    case IMAGE_FOTMAT_48BITS_3COMPONENTS: return 6;
    case IMAGE_FOTMAT_24BITS_RGB:
    case IMAGE_FOTMAT_24BITS_3COMPONENTS: return 3;
    case IMAGE_FOTMAT_64BITS_4COMPONENTS:
    case IMAGE_FOTMAT_64BITS_ARGB: return 8;
    default: return 0;
  }
}

// The reference's picture format (dec_jp2.cpp:488-523): from the component count, the
// component sampling and, for three equally sampled components, the JP2 colour space (16
// sRGB, 18 sYCC) or else the COD transform flag
EncodeFormat encode_format(const j2k::StreamHeader &H) {
  auto sub = [&](const int (&s)[J2K_MAX_COMPONENTS], int a, int b, int c) {
    return s[0] == a && s[1] == b && s[2] == c;
  };
  if (H.ncomp == 1) return H.sub_x[0] == 1 && H.sub_y[0] == 1 ? RAW : UNKNOWN_FORMAT;
  if (H.ncomp == 4) return COMPONENT4;
  if (H.ncomp != 3) return UNKNOWN_FORMAT;
  if (sub(H.sub_x, 1, 2, 2) && sub(H.sub_y, 1, 2, 2)) return YUV420;
  if (sub(H.sub_x, 1, 2, 2) && sub(H.sub_y, 1, 1, 1)) return YUV422;
  if (sub(H.sub_x, 1, 1, 1) && sub(H.sub_y, 1, 2, 2)) return BAYERGRB;
  if (!sub(H.sub_x, 1, 1, 1) || !sub(H.sub_y, 1, 1, 1)) return UNKNOWN_FORMAT;
  if (H.jp2_colr_method == 1 && H.jp2_colr_enum == 16) return RGB;
  if (H.jp2_colr_method == 1 && H.jp2_colr_enum == 18) return YUV444;
  return H.mct ? RGB : YUV444;
}

void fill_props(const j2k::StreamHeader &H, int discard, CodeStreamProperties &P, OutputFormat fmt) {
  std::memset(&P, 0, sizeof(P));
  P.mSize.x = (short)H.image_w();
  P.mSize.y = (short)H.image_h();
  P.mOutputSize.x = (short)H.out_w(discard);
  P.mOutputSize.y = (short)H.out_h(discard);
  P.mThumbOutputSize.x = (short)H.out_w(H.levels[0]);
  P.mThumbOutputSize.y = (short)H.out_h(H.levels[0]);
  P.mOutputFormat = fmt;
  P.mCodeBlockSize.x = (short)(1 << H.cbw_exp[0]);
  P.mCodeBlockSize.y = (short)(1 << H.cbh_exp[0]);
  P.mTileSize.x = (short)H.tile_w;
  P.mTileSize.y = (short)H.tile_h;
  P.mTileNum.x = (short)H.ntx();
  P.mTileNum.y = (short)H.nty();
  P.mComponentNum = (short)H.ncomp;
  P.mCalculatedComponentNum = (short)H.ncomp;
  P.mDwtLevel = (short)H.levels[0];
  P.mLayer = (short)H.layers;
  P.mBitDepth = (short)H.depth[0];
  P.mRoiShift = (short)H.roi_shift[0];
  P.mFormat = encode_format(H);
  P.mMethod = H.reversible[0] ? Ckernels_W5X3 : Ckernels_W9X7;
  P.mProgression = (Jp2_Progression)H.progression;
  P.mHeaderLength = (int)H.header_len;
}

class GpuDecoder : public Decoder {
 public:
  ~GpuDecoder() override {
    if (ctx_) j2k_gpu_ctx_destroy(ctx_);
  }

  int Init(const P_EnginConfig cfg) override {
    std::lock_guard<std::mutex> g(mu_);
    if (cfg) cfg_ = *cfg;
    if (!cfg_.mUsingGpu) return -1;  // no CPU path in this library
    if (cfg_.mOutputQueueLen < 1) cfg_.mOutputQueueLen = 1;
    if (!ctx_) {
      int rc = j2k_gpu_ctx_create(0, 0, &ctx_);
      if (rc != J2K_OK) {
        ctx_ = nullptr;
        return rc;
      }
    }
    slots_.assign(cfg_.mOutputQueueLen, Slot());
    return 0;
  }
  const EnginConfig *GetEngineConfig() const override { return &cfg_; }

  void SetJobConfig(const DecodeJobConfig &c) override { job_ = c; }
  void GetJobConfig(DecodeJobConfig &c, CodeStreamHandler h) const override {
    if (h == INVALID) {
      c = job_;
      return;
    }
    const Slot *s = find(h);
    c = s ? s->cfg : job_;
  }

  Status PreDecode(const void *buf, int size, CodeStreamProperties &props) override {
    if (!buf || size <= 0) return PARSE_ERROR_INVALID_INPUT;
    j2k::StreamHeader H;
    int rc = j2k::parse_header((const uint8_t *)buf, (size_t)size, H);
    if (rc == j2k::PARSE_ERR_UNSUPPORTED) return PARSE_ERROR_UNSUPPORTED_FORMAT;
    if (rc != j2k::PARSE_OK) return PARSE_ERROR;
    fill_props(H, discard_of(H), props, job_.mOutputFormat);
    return READY;
  }

  CodeStreamHandler Decode(const void *buf, int size) override {
    double t;
    return Decode(buf, size, t);
  }

  CodeStreamHandler Decode(const void *buf, int size, double &time) override {
    std::lock_guard<std::mutex> g(mu_);
    time = 0;
    if (!ctx_ || slots_.empty()) return INVALID;
    finish_pending();
    auto t0 = std::chrono::steady_clock::now();
    const CodeStreamHandler h = ++counter_;
    Slot &s = slots_[h % slots_.size()];
    s = Slot();
    s.handler = h;
    s.cfg = job_;
    if (!buf || size <= 0) {
      s.status = PARSE_ERROR_INVALID_INPUT;
      return h;
    }
    s.codestream.assign((const uint8_t *)buf, (const uint8_t *)buf + size);
    j2k::StreamHeader H;
    int prc = j2k::parse_header(s.codestream.data(), s.codestream.size(), H);
    if (prc != j2k::PARSE_OK) {
      s.status = prc == j2k::PARSE_ERR_UNSUPPORTED ? PARSE_ERROR_UNSUPPORTED_FORMAT : PARSE_ERROR;
      return h;
    }
    const int discard = discard_of(H);
    fill_props(H, discard, s.props, s.cfg.mOutputFormat);
    for (int c = 0; c < H.ncomp && c < J2K_MAX_COMPONENTS; ++c) {
      s.comp_w[c] = H.comp_w(c, discard);
      s.comp_h[c] = H.comp_h(c, discard);
    }
    j2k_plan *plan = nullptr;
    int rc = j2k_plan_create_mt(s.codestream.data(), s.codestream.size(), discard, 0, s.cfg.mIgnoreComponents, tier2_threads(),
                                &plan);
    if (rc != J2K_OK) {
      s.status = rc == J2K_ERR_UNSUPPORTED ? PARSE_ERROR_UNSUPPORTED_FORMAT : PARSE_ERROR;
      return h;
    }
    plan_.reset(plan);
    int fmt = fmt_bytes(s.cfg.mOutputFormat) ? (int)s.cfg.mOutputFormat : J2K_FMT_NONE;
    if ((rc = j2k_gpu_batch_begin(ctx_)) != J2K_OK || (rc = j2k_gpu_batch_add(ctx_, plan, fmt, 0, &s.gpu_slot)) != J2K_OK ||
        (rc = bmi_engine::set_checkout(ctx_, s.gpu_slot, s.cfg.mCheckOutComponent)) != J2K_OK ||
        (rc = j2k_gpu_batch_launch(ctx_, nullptr)) != J2K_OK) {
      s.status = DECODE_ERROR;
      return h;
    }
    s.pending = true;
    s.status = DECODING;
    pending_ = h;
    if (cfg_.mSyncMode) finish_pending();
    time = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return h;
  }

  Status CheckStatus(CodeStreamHandler h) const override {
    std::lock_guard<std::mutex> g(mu_);
    const Slot *s = find(h);
    if (!s) return h > 0 && h <= counter_ ? RELEASED : INVALID_STATUS;
    if (s->pending) {
      GpuDecoder *self = const_cast<GpuDecoder *>(this);
      if (j2k_gpu_batch_sync(self->ctx_, 0) == J2K_OK) self->finish_pending();
    }
    return s->status;
  }

  bool CheckProperties(CodeStreamHandler h, CodeStreamProperties &p) const override {
    std::lock_guard<std::mutex> g(mu_);
    const Slot *s = find(h);
    if (!s || s->status == PARSE_ERROR || s->status == PARSE_ERROR_INVALID_INPUT) return false;
    p = s->props;
    return true;
  }

  const void *GetResult(CodeStreamHandler h, int &size) override {
    std::lock_guard<std::mutex> g(mu_);
    size = 0;
    Slot *s = find(h);
    if (!s) return nullptr;
    if (s->pending) finish_pending();
    if (s->status != READY || s->result.empty()) return nullptr;
    size = (int)s->result.size();
    return s->result.data();
  }

  const void *GetThumbnail(CodeStreamHandler h, int &size) override {
    std::lock_guard<std::mutex> g(mu_);
    size = 0;
    Slot *s = find(h);
    if (!s) return nullptr;
    if (s->pending) finish_pending();
    if (s->status != READY) return nullptr;
    if (s->thumb.empty()) {
      int fmt = fmt_bytes(s->cfg.mOutputFormat) ? (int)s->cfg.mOutputFormat : (int)IMAGE_FOTMAT_32BITS_ARGB;
      if (!decode_side(*s, s->props.mDwtLevel, fmt, s->thumb)) return nullptr;
    }
    size = (int)s->thumb.size();
    return s->thumb.data();
  }

  const int *GetDecodedComponentInt(CodeStreamHandler h, int &size, int comp, int tile) override {
    (void)tile;
    std::lock_guard<std::mutex> g(mu_);
    size = 0;
    Slot *s = find(h);
    if (!s || !load_component(*s, comp) || s->props.mMethod != Ckernels_W5X3) return nullptr;
    size = (int)(s->comp_int.size() * sizeof(int));
    return s->comp_int.data();
  }

  const float *GetDecodedComponentFloat(CodeStreamHandler h, int &size, int comp, int tile) override {
    (void)tile;
    std::lock_guard<std::mutex> g(mu_);
    size = 0;
    Slot *s = find(h);
    if (!s || !load_component(*s, comp) || s->props.mMethod != Ckernels_W9X7) return nullptr;
    size = (int)(s->comp_float.size() * sizeof(float));
    return s->comp_float.data();
  }

  void Release(CodeStreamHandler h) override {
    std::lock_guard<std::mutex> g(mu_);
    Slot *s = find(h);
    if (!s) return;
    if (s->pending) finish_pending();
    *s = Slot();
  }

  void GetVersion(int &mainV, int &subV, int &branchV, int &year, int &month, int &date) override {
    mainV = 5;
    subV = 0;
    branchV = 0;
    year = 2026;
    month = 12;
    date = 3;
  }

 private:
  struct PlanDel {
    void operator()(j2k_plan *p) const { j2k_plan_destroy(p); }
  };

  // host threads for the Tier-2 of a multi-tile picture: the engine's worker-thread count
  // (the reference's default of one thread when it is not set)
  int tier2_threads() const { return cfg_.mThreadNum > 1 ? cfg_.mThreadNum : 1; }

  int discard_of(const j2k::StreamHeader &H) const {
    int top = job_.mDwtDecodeTopLevel;
    if (top < 0 || top >= H.levels[0]) return 0;
    return H.levels[0] - top;
  }
  Slot *find(CodeStreamHandler h) {
    if (h <= 0 || slots_.empty()) return nullptr;
    Slot &s = slots_[h % slots_.size()];
    return s.handler == h ? &s : nullptr;
  }
  const Slot *find(CodeStreamHandler h) const { return const_cast<GpuDecoder *>(this)->find(h); }

  void finish_pending() {
    if (pending_ == INVALID) return;
    Slot *s = find(pending_);
    int rc = j2k_gpu_batch_sync(ctx_, -1);
    if (s) {
      s->pending = false;
      if (rc != J2K_OK) {
        s->status = DECODE_ERROR;
      } else {
        int st = j2k_gpu_image_status(ctx_, s->gpu_slot, nullptr);
        const void *d;
        size_t bytes = 0;
        j2k_gpu_output_device(ctx_, s->gpu_slot, &d, &bytes);
        if (bytes) {
          s->result.resize(bytes);
          j2k_gpu_output_copy(ctx_, s->gpu_slot, s->result.data(), bytes);
        }
        s->status = st == J2K_OK ? READY : DECODE_ERROR;
        s->comp_loaded = -1;
        resident_ = s->handler;
      }
    }
    pending_ = INVALID;
  }

  // decode the slot's codestream again with other options into `out`
  bool decode_side(Slot &s, int discard, int fmt, std::vector<uint8_t> &out) {
    finish_pending();
    j2k_plan *p = nullptr;
    if (j2k_plan_create_mt(s.codestream.data(), s.codestream.size(), discard, 0, s.cfg.mIgnoreComponents, tier2_threads(),
                           &p) != J2K_OK)
      return false;
    j2k_image_info I;
    j2k_plan_info(p, &I);
    out.resize(j2k_output_bytes(&I, fmt));
    bool ok = j2k_gpu_batch_begin(ctx_) == J2K_OK && j2k_gpu_batch_add(ctx_, p, fmt, 0, nullptr) == J2K_OK &&
              j2k_gpu_batch_launch(ctx_, nullptr) == J2K_OK && j2k_gpu_batch_sync(ctx_, -1) == J2K_OK &&
              j2k_gpu_output_copy(ctx_, 0, out.data(), out.size()) == J2K_OK;
    j2k_plan_destroy(p);
    resident_ = INVALID;
    return ok;
  }

  bool load_component(Slot &s, int comp) {
    if (s.pending) finish_pending();
    if (s.status != READY || comp < 0 || comp >= s.props.mComponentNum) return false;
    if (s.comp_loaded == comp) return true;
    // decode the picture again with its components kept (when the device buffers hold
    // another picture, or this picture's packed decode fused its last level with the output)
    auto redecode = [&]() {
      finish_pending();
      j2k_plan *p = nullptr;
      if (j2k_plan_create_mt(s.codestream.data(), s.codestream.size(), discard_of_slot(s), 0, s.cfg.mIgnoreComponents,
                             tier2_threads(), &p) != J2K_OK)
        return false;
      plan_.reset(p);
      if (j2k_gpu_batch_begin(ctx_) != J2K_OK || j2k_gpu_batch_add(ctx_, p, J2K_FMT_NONE, 0, &s.gpu_slot) != J2K_OK ||
          j2k_gpu_batch_launch(ctx_, nullptr) != J2K_OK || j2k_gpu_batch_sync(ctx_, -1) != J2K_OK)
        return false;
      resident_ = s.handler;
      return true;
    };
    if (resident_ != s.handler && !redecode()) return false;
    // the component on its own grid: sub-sampled components are smaller than the picture
    const size_t n = (size_t)s.comp_w[comp] * s.comp_h[comp];
    void *dst;
    if (s.props.mMethod == Ckernels_W5X3) {
      s.comp_int.resize(n);
      dst = s.comp_int.data();
    } else {
      s.comp_float.resize(n);
      dst = s.comp_float.data();
    }
    int rc = j2k_gpu_component_copy(ctx_, s.gpu_slot, comp, dst, n * 4);
    if (rc == J2K_ERR_STATE) {
      if (!redecode()) return false;
      rc = j2k_gpu_component_copy(ctx_, s.gpu_slot, comp, dst, n * 4);
    }
    if (rc != J2K_OK) return false;
    s.comp_loaded = comp;
    return true;
  }
  int discard_of_slot(const Slot &s) const {
    int top = s.cfg.mDwtDecodeTopLevel;
    if (top < 0 || top >= s.props.mDwtLevel) return 0;
    return s.props.mDwtLevel - top;
  }

  mutable std::mutex mu_;
  EnginConfig cfg_;
  DecodeJobConfig job_;
  j2k_gpu_ctx *ctx_ = nullptr;
  std::vector<Slot> slots_;
  CodeStreamHandler counter_ = 0;
  CodeStreamHandler pending_ = INVALID;
  CodeStreamHandler resident_ = INVALID;
  std::unique_ptr<j2k_plan, PlanDel> plan_;
};

GpuDecoder *g_decoder = nullptr;
std::mutex g_mu;

}  // namespace

namespace BMI {
Decoder *Decoder::Get() {
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_decoder) g_decoder = new (std::nothrow) GpuDecoder();
  return g_decoder;
}
void Decoder::Terminate() {
  std::lock_guard<std::mutex> g(g_mu);
  delete g_decoder;
  g_decoder = nullptr;
}
}  // namespace BMI

// ---------------------------------------------------------------- C binding ------------
// A C surface over the singleton for FFI callers (ctypes, cgo, JNI) that cannot call C++
// virtual functions; each call maps one-to-one onto a BMI::Decoder method.
extern "C" {

int bmi_decoder_init(int sync_mode, int output_queue_len) {
  BMI::Decoder *d = BMI::Decoder::Get();
  if (!d) return -1;
  BMI::EnginConfig c;
  c.mSyncMode = sync_mode != 0;
  c.mOutputQueueLen = output_queue_len > 0 ? output_queue_len : 1;
  return d->Init(&c);
}
void bmi_decoder_set_job(int output_format, int dwt_top_level, unsigned ignore_components, int checkout_component) {
  BMI::DecodeJobConfig j;
  j.mOutputFormat = (OutputFormat)output_format;
  j.mDwtDecodeTopLevel = dwt_top_level;
  j.mIgnoreComponents = ignore_components;
  j.mCheckOutComponent = checkout_component;
  BMI::Decoder::Get()->SetJobConfig(j);
}
int bmi_decoder_decode(const void *buf, int size, double *ms) {
  double t = 0;
  int h = BMI::Decoder::Get()->Decode(buf, size, t);
  if (ms) *ms = t;
  return h;
}
int bmi_decoder_predecode(const void *buf, int size, int *width, int *height, int *ncomp, int *bitdepth, int *levels) {
  BMI::CodeStreamProperties p;
  BMI::Status s = BMI::Decoder::Get()->PreDecode(buf, size, p);
  if (s == BMI::READY) {
    if (width) *width = p.mSize.x;
    if (height) *height = p.mSize.y;
    if (ncomp) *ncomp = p.mComponentNum;
    if (bitdepth) *bitdepth = p.mBitDepth;
    if (levels) *levels = p.mDwtLevel;
  }
  return (int)s;
}
int bmi_decoder_predecode_format(const void *buf, int size, int *format, int *method) {
  BMI::CodeStreamProperties p;
  BMI::Status s = BMI::Decoder::Get()->PreDecode(buf, size, p);
  if (s == BMI::READY) {
    if (format) *format = (int)p.mFormat;
    if (method) *method = (int)p.mMethod;
  }
  return (int)s;
}
int bmi_decoder_status(int h) { return (int)BMI::Decoder::Get()->CheckStatus(h); }
const void *bmi_decoder_result(int h, int *size) {
  int s = 0;
  const void *p = BMI::Decoder::Get()->GetResult(h, s);
  if (size) *size = s;
  return p;
}
const void *bmi_decoder_thumbnail(int h, int *size) {
  int s = 0;
  const void *p = BMI::Decoder::Get()->GetThumbnail(h, s);
  if (size) *size = s;
  return p;
}
const int *bmi_decoder_component_int(int h, int comp, int *size) {
  int s = 0;
  const int *p = BMI::Decoder::Get()->GetDecodedComponentInt(h, s, comp);
  if (size) *size = s;
  return p;
}
const float *bmi_decoder_component_float(int h, int comp, int *size) {
  int s = 0;
  const float *p = BMI::Decoder::Get()->GetDecodedComponentFloat(h, s, comp);
  if (size) *size = s;
  return p;
}
void bmi_decoder_release(int h) { BMI::Decoder::Get()->Release(h); }
void bmi_decoder_terminate(void) { BMI::Decoder::Terminate(); }
}
