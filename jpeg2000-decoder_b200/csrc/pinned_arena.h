/*
 * pinned_arena.h — page-locked host memory for decoded pictures, carved from large chunks.
 *
 * Page-locking costs far more than a copy (about 13 ms for a 4K 8-bit picture), so the
 * service keeps its output buffers.  A pool of per-request buffers reuses a buffer only for
 * a request of about its size, so a stream of mixed sizes keeps allocating whenever one
 * size runs short although larger or smaller buffers sit free.  The arena instead takes
 * chunks of at least CHUNK bytes and hands out best-fitting pieces of them; a released piece
 * merges with free neighbours of the same chunk, so free memory serves any size and the
 * arena stops growing once it covers the peak of bytes held at once.
 *
 * Host code only; the page-locking functions are template parameters (cudaMallocHost /
 * cudaFreeHost in the service, malloc / free in the unit test).  Thread-safe.
 */
#ifndef J2K_PINNED_ARENA_H
#define J2K_PINNED_ARENA_H

#include <cstddef>
#include <cstdint>
#include <iterator>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace j2k {

template <class Alloc, class Free>
class PinnedArena {
 public:
  static constexpr size_t CHUNK = size_t(256) << 20;  // bytes page-locked at a time (at least)
  static constexpr size_t ALIGN = 4096;               // piece granularity and alignment

  PinnedArena(Alloc a, Free f) : alloc_(a), free_(f) {}
  ~PinnedArena() {
    for (const Chunk &c : chunks_) free_(c.base);
  }
  PinnedArena(const PinnedArena &) = delete;
  PinnedArena &operator=(const PinnedArena &) = delete;

  // A piece of at least n bytes, or nullptr when page-locking fails.  *grew is set when a
  // new chunk had to be page-locked for it.
  uint8_t *get(size_t n, bool *grew) {
    *grew = false;
    n = n ? (n + ALIGN - 1) / ALIGN * ALIGN : ALIGN;
    std::lock_guard<std::mutex> lk(mu_);
    uint8_t *p = take(n);
    if (p) return p;
    const size_t cap = n > CHUNK ? n : CHUNK;
    uint8_t *base = static_cast<uint8_t *>(alloc_(cap));
    if (!base) return nullptr;
    *grew = true;
    chunks_.push_back({base, cap});
    free_by_addr_[base] = {cap, chunks_.size() - 1};
    return take(n);
  }

  // Return a piece obtained from get (nullptr is ignored).
  void put(uint8_t *p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu_);
    auto it = used_.find(p);
    if (it == used_.end()) return;
    Piece piece = it->second;
    used_.erase(it);
    // merge with the free piece that ends at p and the one that starts after it (same chunk)
    auto next = free_by_addr_.lower_bound(p);
    if (next != free_by_addr_.end() && next->first == p + piece.size && next->second.chunk == piece.chunk) {
      piece.size += next->second.size;
      next = free_by_addr_.erase(next);
    }
    if (next != free_by_addr_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second.size == p && prev->second.chunk == piece.chunk) {
        prev->second.size += piece.size;
        return;
      }
    }
    free_by_addr_[p] = piece;
  }

  size_t reserved_bytes() const {
    std::lock_guard<std::mutex> lk(mu_);
    size_t s = 0;
    for (const Chunk &c : chunks_) s += c.size;
    return s;
  }
  size_t chunks() const {
    std::lock_guard<std::mutex> lk(mu_);
    return chunks_.size();
  }

 private:
  struct Chunk {
    uint8_t *base;
    size_t size;
  };
  struct Piece {
    size_t size;
    size_t chunk;
  };

  // best fit among the free pieces (the smallest that holds n), split off the front
  uint8_t *take(size_t n) {
    auto best = free_by_addr_.end();
    for (auto it = free_by_addr_.begin(); it != free_by_addr_.end(); ++it)
      if (it->second.size >= n && (best == free_by_addr_.end() || it->second.size < best->second.size)) best = it;
    if (best == free_by_addr_.end()) return nullptr;
    uint8_t *p = best->first;
    const Piece f = best->second;
    free_by_addr_.erase(best);
    if (f.size > n) free_by_addr_[p + n] = {f.size - n, f.chunk};
    used_[p] = {n, f.chunk};
    return p;
  }

  Alloc alloc_;
  Free free_;
  mutable std::mutex mu_;
  std::vector<Chunk> chunks_;
  std::map<uint8_t *, Piece> free_by_addr_;
  std::unordered_map<uint8_t *, Piece> used_;
};

}  // namespace j2k

#endif
