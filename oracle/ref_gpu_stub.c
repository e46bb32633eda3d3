/*
 * ref_gpu_stub.c — the reference's CUDA-1.0 kernel launchers (decoder/cudainterface/src/
 * gpufunc.h; implemented in gpufunc.cu with legacy texture references, which CUDA 12 no
 * longer compiles) replaced by functions that report "no GPU".  The reference engine then
 * runs its CPU DWT path (decoderconcrete.cpp:195-218).  TEST AND BASELINE INFRASTRUCTURE
 * ONLY (oracle/build_ref_cpu.sh); compiled as C++ so the C prototypes link as extern "C".
 */
#include "gpufunc.h"

extern "C" {
int bmi_get_gpu_info(GpuInfo *gpu) { (void)gpu; return -1; }
int bmi_del_gpu_info(GpuInfo *gpu) { (void)gpu; return 0; }
void malloc_gpu_buf(CudaBuf *buf) { (void)buf; }
void delete_gpu_buf(CudaBuf *buf) { (void)buf; }
StreamId bmi_gpu_stream_new() { return (StreamId)0; }
void bmi_gpu_stream_delete(StreamId *s) { (void)s; }
void bmi_sync_job(StreamId *s) { (void)s; }
int memory_copy_2D(void *d, size_t dp, void *s, size_t sp, size_t w, size_t h, StreamId *a, int dir) { return -1; }
int memory_copy_linear(void *d, void *s, int n, StreamId a, int dir) { return -1; }
void bmi_idwt_r53_gpu_transform(TileInfo_c *t, CompInfo_c *c, CudaBuf *o, CudaBuf *tmp, StreamId a, short w, int top) {}
void bmi_idwt_i97_gpu_transform_float(TileInfo_c *t, CompInfo_c *c, CudaBuf *o, CudaBuf *tmp, StreamId a, short w, int top) {}
int bmi_MCT_gpu(TileInfo_c *t, int bd, int ws, int dl, int decl, int epp, int bpe, StreamId a) { return -1; }
int bmi_ICT_gpu(TileInfo_c *t, int bd, int ws, int dl, int decl, int epp, int bpe, StreamId a) { return -1; }
int bmi_merge_gpu(TileInfo_c *t, int cn, int dl, int decl, short bd, short ws, int ip, int epp, int bpe, EncodeMathod m,
                  StreamId a) { return -1; }
int bmi_get_one_component(TileInfo_c *t, int c, EncodeMathod m, int mct, int bd, int ws, int decl, StreamId a) { return -1; }
int bmi_get_one_component_orig(TileInfo_c *t, int c, EncodeMathod m, int bd, int ws, int decl, StreamId a) { return -1; }
int bmi_dc_shift(CudaBuf *cb, CudaBuf *ct, int sx, int sy, int dx, int dy, int w, int h, int wl, int bd, int f, StreamId a) {
  return -1;
}
void bmi_idwt_i97_gpu_transform_resolution(CudaBuf *o, CudaBuf *t, int x, int y, int lw, int hw, int lh, int hh, int xp,
                                           int yp, float c0, float c1, float c2, float c3, int ll, short wl, StreamId a) {}
void bmi_idwt_r53_gpu_transform_resolution(CudaBuf *o, CudaBuf *t, int x, int y, int lw, int hw, int lh, int hh, int xp,
                                           int yp, int ll, short wl, StreamId a) {}
}
