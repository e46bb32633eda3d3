/*
 * Seeded corruption driver for the host Tier-2 (j2k_plan_create_mt), built with
 * AddressSanitizer and UndefinedBehaviorSanitizer by tests/test_cpu_tier2.py: every seed
 * codestream in the directory argv[1] is mutated (bytes flipped in the headers or anywhere,
 * truncated, runs inserted or deleted) argv[3] times from the seed argv[2], planned at full
 * or reduced resolution on one or three threads, and destroyed.  A sanitizer report ends the
 * process with a non-zero status.
 */
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <dirent.h>
#include <random>
#include <string>
#include <vector>
#include "j2k_gpu.h"
int main(int argc, char **argv) {
  std::vector<std::vector<unsigned char>> seeds;
  DIR *d = opendir(argv[1]);
  for (dirent *e; (e = readdir(d));) {
    std::string n = e->d_name;
    if (n.size() < 5 || n.substr(n.size() - 4) != ".j2k") continue;
    FILE *f = fopen((std::string(argv[1]) + "/" + n).c_str(), "rb");
    fseek(f, 0, SEEK_END); long len = ftell(f); fseek(f, 0, SEEK_SET);
    std::vector<unsigned char> b(len); if (fread(b.data(), 1, len, f) != (size_t)len) return 2; fclose(f);
    if (len >= 16 && len < 400000) seeds.push_back(b);
  }
  closedir(d);
  if (seeds.empty()) return 2;
  std::mt19937_64 rng(atoi(argv[2]));
  const int N = atoi(argv[3]);
  int ok = 0, bad = 0;
  for (int it = 0; it < N; ++it) {
    std::vector<unsigned char> cs = seeds[rng() % seeds.size()];
    int muts = 1 + rng() % 3;
    for (int m = 0; m < muts; ++m) {
      int k = rng() % 5;
      if (k == 0) cs[rng() % std::min<size_t>(cs.size(), 600)] = rng() & 255;
      else if (k == 1) { int c = 1 + rng() % 16; for (int i = 0; i < c; ++i) cs[rng() % cs.size()] = rng() & 255; }
      else if (k == 2) { if (cs.size() > 2) cs.resize(2 + rng() % (cs.size() - 2)); }
      else if (k == 3) { size_t j = rng() % cs.size(); int c = 1 + rng() % 8; for (int i = 0; i < c; ++i) cs.insert(cs.begin() + j, rng() & 255); }
      else { size_t j = rng() % cs.size(); size_t c = std::min<size_t>(1 + rng() % 8, cs.size() - j); if (cs.size() - c >= 2) cs.erase(cs.begin() + j, cs.begin() + j + c); }
    }
    j2k_plan *p = nullptr;
    int threads = (rng() % 3 == 0) ? 3 : 1;
    if (j2k_plan_create_mt(cs.data(), cs.size(), (int)(rng() % 3), 0, 0, threads, &p) == J2K_OK) { ++ok; j2k_plan_destroy(p); }
    else ++bad;
  }
  printf("asan fuzz seed %s: planned %d refused %d\n", argv[2], ok, bad);
}
