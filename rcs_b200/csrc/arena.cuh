// Best-fit sub-allocator over large device chunks, for the context's
// allocations of 256 KB and more (see DevBuf::alloc).
//
// The factorization allocates and frees hundreds of thousands of blocks of
// every size; each stream-ordered pool call for a large block costs tens of
// microseconds to milliseconds of host time.  The arena carves such blocks
// out of chunks it keeps -- 64 MB at first, each new chunk as large as all
// earlier ones together up to 512 MB (so a small body's context, one of a
// batch of dozens, holds little), or one request's size when larger: a free
// block is found by size in a multimap, split, and merged with its free
// neighbours of the same chunk when released.  Every use of context memory
// is ordered on the context's one stream, so a released range can be handed
// out again at once.
//
// This header is pure host arithmetic on addresses (no CUDA calls): the chunk
// source is a callback, which lets the CPU tests drive it with fake
// addresses.
#pragma once
#include <cstddef>
#include <cstdint>
#include <functional>
#include <map>
#include <vector>

namespace aifmm {

class Arena {
 public:
  static constexpr size_t kAlign = 512;
  static constexpr size_t kChunk = (size_t)512 << 20;     // largest growth step
  static constexpr size_t kFirstChunk = (size_t)64 << 20;  // first growth step
  static constexpr size_t kMinSize = (size_t)256 << 10;

  // grow(bytes) returns the base address of a new chunk of `bytes` bytes, or 0.
  explicit Arena(std::function<uint64_t(size_t)> grow) : grow_(std::move(grow)) {}

  static size_t round(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

  // Address of a free range of at least n bytes, or 0 when no chunk can be had.
  uint64_t alloc(size_t n) {
    const size_t need = round(n == 0 ? 1 : n);
    auto it = bySize_.lower_bound(need);
    if (it == bySize_.end()) {
      // geometric growth: as much as the chunks held so far, at least the first step, at most kChunk
      const size_t step = bytesHeld_ < kFirstChunk ? kFirstChunk : (bytesHeld_ > kChunk ? kChunk : bytesHeld_);
      const size_t bytes = need > step ? need : step;
      const uint64_t base = grow_(bytes);
      if (base == 0) return 0;
      chunks_[base] = bytes;
      bytesHeld_ += bytes;
      insertFree(base, bytes);
      it = bySize_.lower_bound(need);
    }
    const size_t size = it->first;
    const uint64_t addr = it->second;
    bySize_.erase(it);
    byAddr_.erase(addr);
    if (size > need) insertFree(addr + need, size - need);
    used_[addr] = need;
    bytesUsed_ += need;
    return addr;
  }

  // Returns the range that alloc handed out at addr; false if addr is not one.
  bool release(uint64_t addr) {
    auto u = used_.find(addr);
    if (u == used_.end()) return false;
    size_t size = u->second;
    used_.erase(u);
    bytesUsed_ -= size;
    uint64_t start = addr;
    const uint64_t chunk = chunkOf(addr);
    // merge with the free range that ends here and the one that starts after
    auto next = byAddr_.find(start + size);
    if (next != byAddr_.end() && chunkOf(next->first) == chunk) {
      eraseFree(next->first, next->second);
      size += next->second;
    }
    auto prev = byAddr_.lower_bound(start);
    if (prev != byAddr_.begin()) {
      --prev;
      if (prev->first + prev->second == start && chunkOf(prev->first) == chunk) {
        const uint64_t pa = prev->first;
        const size_t ps = prev->second;
        eraseFree(pa, ps);
        start = pa;
        size += ps;
      }
    }
    insertFree(start, size);
    return true;
  }

  // Chunks with nothing allocated in them, removed from the arena (their
  // memory can go back to the device).
  std::vector<std::pair<uint64_t, size_t>> takeFreeChunks() {
    std::vector<std::pair<uint64_t, size_t>> out;
    for (auto c = chunks_.begin(); c != chunks_.end();) {
      auto f = byAddr_.find(c->first);
      if (f != byAddr_.end() && f->second == c->second) {
        eraseFree(f->first, f->second);
        out.push_back(*c);
        bytesHeld_ -= c->second;
        c = chunks_.erase(c);
      } else {
        ++c;
      }
    }
    return out;
  }

  std::vector<std::pair<uint64_t, size_t>> chunks() const { return {chunks_.begin(), chunks_.end()}; }
  size_t bytesUsed() const { return bytesUsed_; }
  size_t freeRanges() const { return byAddr_.size(); }
  bool owns(uint64_t addr) const { return used_.count(addr) != 0; }

 private:
  uint64_t chunkOf(uint64_t addr) const {
    auto c = chunks_.upper_bound(addr);
    --c;  // every address handed out lies in a chunk
    return c->first;
  }
  void insertFree(uint64_t addr, size_t size) {
    byAddr_[addr] = size;
    bySize_.insert({size, addr});
  }
  void eraseFree(uint64_t addr, size_t size) {
    byAddr_.erase(addr);
    auto r = bySize_.equal_range(size);
    for (auto it = r.first; it != r.second; ++it)
      if (it->second == addr) {
        bySize_.erase(it);
        break;
      }
  }
  std::function<uint64_t(size_t)> grow_;
  std::map<uint64_t, size_t> chunks_;   // base -> bytes
  std::map<uint64_t, size_t> byAddr_;   // free ranges by address
  std::multimap<size_t, uint64_t> bySize_;
  std::map<uint64_t, size_t> used_;     // handed-out ranges
  size_t bytesUsed_ = 0;
  size_t bytesHeld_ = 0;  // bytes of all chunks held
};

}  // namespace aifmm
