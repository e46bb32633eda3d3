// CPU unit test of the service's pinned output arena (jpeg2000-decoder_b200/csrc/
// pinned_arena.h) with malloc / free standing in for page-locking.  Prints one line per
// check and exits non-zero on the first failure.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <vector>

#include "../jpeg2000-decoder_b200/csrc/pinned_arena.h"

namespace {
int g_allocs = 0;
void *test_alloc(size_t n) {
  g_allocs++;
  // 4096-aligned like page-locked memory
  void *p = nullptr;
  return posix_memalign(&p, 4096, n) == 0 ? p : nullptr;
}
void test_free(void *p) { std::free(p); }
typedef j2k::PinnedArena<void *(*)(size_t), void (*)(void *)> Arena;

int fail(const char *what) {
  std::printf("FAIL %s\n", what);
  return 1;
}
}  // namespace

int main() {
  const size_t MB = size_t(1) << 20;
  // sizes of decoded pictures in the service's mix: 256^2 .. 4096x2160, 8 and 16 bits
  const size_t sizes[] = {196608, 786432, 3145728, 6220800, 26542080, 53084160, 1048576 * 3 / 2, 12 * MB};
  std::mt19937 rng(7);
  {
    Arena a(test_alloc, test_free);
    std::map<uint8_t *, size_t> live;  // start -> bytes requested
    int grew_late = 0;
    for (int step = 0; step < 20000; ++step) {
      const bool take = live.size() < 40 && (live.empty() || rng() % 2);
      if (take) {
        const size_t n = sizes[rng() % 8];
        bool grew = false;
        uint8_t *p = a.get(n, &grew);
        if (!p) return fail("get returned nullptr");
        if ((uintptr_t)p % Arena::ALIGN) return fail("piece not aligned");
        // no overlap with any live piece
        auto it = live.upper_bound(p);
        if (it != live.end() && p + n > it->first) return fail("overlaps the next live piece");
        if (it != live.begin()) {
          auto pv = std::prev(it);
          if (pv->first + pv->second > p) return fail("overlaps the previous live piece");
        }
        live[p] = n;
        if (grew && step > 5000) grew_late++;
      } else {
        auto it = live.begin();
        std::advance(it, rng() % live.size());
        a.put(it->first);
        live.erase(it);
      }
    }
    // at most 40 pieces of <= 53 MB are held at once: the arena stops growing early
    std::printf("chunks %zu, reserved %zu MB, growth after step 5000: %d\n", a.chunks(), a.reserved_bytes() / MB,
                grew_late);
    if (grew_late > 2) return fail("arena kept growing in steady state");
    for (auto &kv : live) a.put(kv.first);
    // everything released: each chunk is one free piece again, so a whole chunk fits
    const int before = g_allocs;
    std::vector<uint8_t *> whole;
    for (size_t i = 0; i < a.chunks(); ++i) {
      bool grew = false;
      uint8_t *p = a.get(Arena::CHUNK, &grew);
      if (!p || grew) return fail("released pieces did not merge back into whole chunks");
      whole.push_back(p);
    }
    if (g_allocs != before) return fail("allocation while whole chunks were free");
    for (uint8_t *p : whole) a.put(p);
    a.put(nullptr);  // ignored
    std::printf("merge ok\n");
  }
  {
    // a piece larger than a chunk gets a chunk of its own size
    Arena a(test_alloc, test_free);
    bool grew = false;
    uint8_t *p = a.get(Arena::CHUNK + 5 * MB, &grew);
    if (!p || !grew || a.reserved_bytes() < Arena::CHUNK + 5 * MB) return fail("oversized piece");
    a.put(p);
    std::printf("oversized ok\n");
  }
  std::printf("ALL OK\n");
  return 0;
}
