/*
 * A plain C99 caller of the library's C ABI (include/j2k_gpu.h), compiled and run by
 * tests/test_cpu_tier2.py: it is what a cgo / FFI / JNI binding sees.  Plans a codestream
 * on the host (no device needed), reads the plan back, and checks the error paths.
 *
 *   c_abi_consumer <codestream.j2k>   -> prints "width height ncomp cblks coded_bytes ctx"
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bmi_decoder_c.h"
#include "bmi_jp2dec.h"
#include "j2k_gpu.h"
#include "j2k_server.h"

static int fail(const char *what, int rc) {
  fprintf(stderr, "%s: %d (%s)\n", what, rc, j2k_status_string(rc));
  return 1;
}

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 2;
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  unsigned char *cs = (unsigned char *)malloc((size_t)n);
  if (!cs || fread(cs, 1, (size_t)n, f) != (size_t)n) return 2;
  fclose(f);

  j2k_plan *plan = NULL, *plan3 = NULL;
  int rc = j2k_plan_create(cs, (size_t)n, 0, 0, 0, &plan);
  if (rc != J2K_OK) return fail("j2k_plan_create", rc);
  rc = j2k_plan_create_mt(cs, (size_t)n, 0, 0, 0, 3, &plan3);
  if (rc != J2K_OK) return fail("j2k_plan_create_mt", rc);
  j2k_image_info info, info3;
  if ((rc = j2k_plan_info(plan, &info)) != J2K_OK) return fail("j2k_plan_info", rc);
  if ((rc = j2k_plan_info(plan3, &info3)) != J2K_OK) return fail("j2k_plan_info", rc);
  if (memcmp(&info, &info3, sizeof(info)) != 0) return fail("threaded plan differs", -100);
  if (memcmp(j2k_plan_cblks(plan), j2k_plan_cblks(plan3), (size_t)info.num_cblks * sizeof(j2k_cblk)) != 0 ||
      memcmp(j2k_plan_bytes(plan), j2k_plan_bytes(plan3), (size_t)info.coded_bytes) != 0)
    return fail("threaded plan differs", -101);
  if (!j2k_plan_tilecomps(plan) || info.num_tilecomps < 1) return fail("tilecomps", -102);
  if (j2k_output_bytes(&info, J2K_FMT_24BITS_RGB) != (size_t)info.width * info.height * 3)
    return fail("j2k_output_bytes", -103);

  /* error paths: no plan for garbage, no output for a null plan */
  j2k_plan *bad = NULL;
  static const unsigned char junk[16] = {0xFF, 0x4F, 0xFF, 0x51, 0x00, 0x02};
  if (j2k_plan_create(junk, sizeof(junk), 0, 0, 0, &bad) == J2K_OK || bad) return fail("junk accepted", -104);
  if (j2k_plan_info(NULL, &info3) != J2K_ERR_ARG) return fail("null plan", -105);

  /* a device context: J2K_ERR_NODEVICE without a GPU (there is no CPU path) */
  j2k_gpu_ctx *ctx = NULL;
  const int crc = j2k_gpu_ctx_create(0, 0, &ctx);
  if (ctx) j2k_gpu_ctx_destroy(ctx);

  printf("%d %d %d %d %llu %d\n", info.width, info.height, info.ncomp, info.num_cblks,
         (unsigned long long)info.coded_bytes, crc);
  j2k_plan_destroy(plan);
  j2k_plan_destroy(plan3);
  free(cs);
  return 0;
}
