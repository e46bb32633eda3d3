// Host build of the one-block-per-lane Tier-1 machine (jpeg2000-decoder_b200/csrc/
// t1_lanes.cuh), for the CPU tests: decodes one code-block with the same Lane functions the
// device kernel runs, one lane of the interleaved state, into raw sign-magnitude samples.
#include <cstring>
#include <vector>

#include "../jpeg2000-decoder_b200/csrc/t1_lanes.cuh"

using namespace j2k_lanes;

namespace {
LaneTables g_tables;
bool g_ready = false;
unsigned long long g_steps = 0;
}  // namespace

extern "C" unsigned long long lanes_host_steps() { return g_steps; }

extern "C" int lanes_host_eligible(const j2k_cblk *cb) { return lane_eligible(*cb) ? 1 : 0; }

// Decodes `cb` into out (cb->w * cb->h samples, row-major): returns the block status, or -1
// for a block the lane form does not take.  The other lanes' state is filled with garbage
// so a lane that reads outside its own slots shows up as a mismatch.
extern "C" int lanes_host_block(const j2k_cblk *cb, const uint8_t *bytes, const uint32_t *seglens, int32_t *out) {
  if (!g_ready) {
    build_lane_tables(g_tables);
    g_ready = true;
  }
  if (!lane_eligible(*cb)) return -1;
  std::vector<uint64_t> state((size_t)STATE_U64 * LANES, 0x5A5A5A5A5A5A5A5Aull);
  std::vector<uint32_t> cx((size_t)N_CTX * LANES, 0xA5A5A5A5u);
  const int lane = 7;
  for (int e = 0; e < STATE_U64; ++e) state[(size_t)e * LANES + lane] = 0;
  LaneMem M;
  M.sig = state.data();
  M.chi = M.sig + MAXW * LANES;
  M.pi = M.chi + MAXW * LANES;
  M.rho = M.pi + MAXW * LANES;
  M.nb = M.rho + MAXW * LANES;
  M.sc = M.nb + MAXS * LANES;
  M.cx = cx.data();
  M.lane = lane;
  j2k_cblk c = *cb;
  c.out_stride = c.w;
  std::memset(out, 0, sizeof(int32_t) * c.w * c.h);
  Lane L;
  std::memset(&L, 0, sizeof(L));
  lane_begin(L, M, g_tables, c, bytes, seglens, out);
  while (L.kind != K_DONE) {
    lane_step(L, M, g_tables);
    g_steps++;
  }
  return L.status;
}
