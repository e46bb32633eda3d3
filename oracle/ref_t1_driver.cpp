/*
 * ref_t1_driver.cpp — C entry point into the reference's own Tier-1 block decoder
 * (decode_code_block, decoder/codec/src/bmi_block_decoder.cpp:589-853), compiled from the
 * reference tree in place by oracle/build_ref.sh into oracle/_ref/libref_t1.so.
 * TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle restatement.
 *
 * The reference takes its coded bytes through a per-layer pass list (stru_coding_pass,
 * decoder/codec/include/dec_stru.h:194-221).  Here every pass gets its own one-pass
 * "layer"; the first one points at all of the block's bytes and every cumlen equals the
 * total, so the reference's copy loop (bmi_block_decoder.cpp:744-760) gathers exactly the
 * block's bytes whatever its segment count.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdarg.h>

#include "bmi_block_decoder.h"
#include "dec_stru.h"
#include "dec_t1.h"

extern "C" void dbg_write_log(const char *, ...) {}

extern "C" int ref_t1_block(int w, int h, int missing, int num_pass, int numbps, int band, const uint8_t *data,
                            int data_len, int32_t *out) {
  if (w <= 0 || h <= 0 || w > 1024 || h > 1024 || data_len < 0 || data_len > 65535 || num_pass > 255) return -100;
  int stripes = (h + 3) >> 2;
  int gap = w + 3;
  int32_t *samples = (int32_t *)calloc((size_t)stripes * 4 * w + 16, 4);
  int32_t *ctx = (int32_t *)calloc((size_t)(stripes + 4) * gap + 16, 4);
  uint8_t *pass_buf = (uint8_t *)calloc((size_t)data_len + 16, 1);
  uint8_t *src = (uint8_t *)calloc((size_t)data_len + 16, 1);
  stru_coding_pass *passes = (stru_coding_pass *)calloc((size_t)num_pass + 1, sizeof(stru_coding_pass));
  if (!samples || !ctx || !pass_buf || !src || !passes) return -101;
  memcpy(src, data, (size_t)data_len);
  for (int k = 0; k < num_pass; ++k) {
    passes[k].cumlen = (unsigned short)data_len;
    passes[k].buffer = src;
    passes[k].layer = 0;
    passes[k].num_t2layer = 1;
  }
  stru_code_block cb;
  memset(&cb, 0, sizeof(cb));
  cb.width = (short)w;
  cb.height = (short)h;
  cb.missing_bit_plan = (unsigned char)missing;
  cb.num_pass = (unsigned char)num_pass;
  cb.pass = passes;
  unsigned char *lut = lut_ctx_lllh;
  if (band == 1) lut = lut_ctx_hl;
  if (band == 3) lut = lut_ctx_hh;
  int rc = decode_code_block(false, samples, ctx, pass_buf, numbps, &cb, lut);
  for (int y = 0; y < h; ++y) memcpy(out + (size_t)y * w, samples + (size_t)y * w, sizeof(int32_t) * w);
  free(samples);
  free(ctx);
  free(pass_buf);
  free(src);
  free(passes);
  return rc;
}
