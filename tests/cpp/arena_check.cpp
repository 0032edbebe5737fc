// Randomised checks of the device sub-allocator's bookkeeping
// (rcs_b200/csrc/arena.cuh) with fake chunk addresses: handed-out ranges lie
// inside one chunk, never overlap, are aligned; released ranges merge back so
// that an emptied arena hands every chunk back whole; chunks that happen to be
// adjacent in the address space are never merged; chunks handed back while
// other chunks still hold ranges contain no live range and are never handed
// out again.  The growth policy: 64 MB first, then as much as the arena holds,
// at most 512 MB a step, and one request's size when it is larger.  Exit 0
// and "OK" on success.
#include <cstdio>
#include <map>
#include <random>
#include <vector>

#include "../../rcs_b200/csrc/arena.cuh"

using aifmm::Arena;

static int fails = 0;
#define CHECK(c)                                                    \
  do {                                                              \
    if (!(c)) {                                                     \
      std::printf("FAILED line %d: %s\n", __LINE__, #c);            \
      if (++fails > 10) return 1;                                   \
    }                                                               \
  } while (0)

int main() {
  std::mt19937_64 rng(12345);
  uint64_t next = (uint64_t)1 << 40;
  int grows = 0;
  Arena a([&](size_t bytes) -> uint64_t {
    // every other chunk starts right where the previous one ended
    const uint64_t base = next;
    next += bytes + ((grows++ % 2) ? 0 : (uint64_t)1 << 21);
    return base;
  });
  std::map<uint64_t, size_t> live;  // addr -> requested bytes
  auto inChunk = [&](uint64_t addr, size_t n) {
    for (auto& c : a.chunks())
      if (addr >= c.first && addr + n <= c.first + c.second) return true;
    return false;
  };
  for (int step = 0; step < 60000; ++step) {
    const bool doAlloc = live.empty() || (rng() % 100) < 55;
    if (doAlloc) {
      // sizes from 256 KB to 1.5 GB, log-uniform
      const double e = 18.0 + (rng() % 10000) / 10000.0 * 12.6;
      const size_t n = (size_t)std::exp2(e);
      const uint64_t p = a.alloc(n);
      CHECK(p != 0);
      CHECK(p % Arena::kAlign == 0);
      CHECK(inChunk(p, Arena::round(n)));
      auto after = live.lower_bound(p);
      if (after != live.end()) CHECK(p + Arena::round(n) <= after->first);
      if (after != live.begin()) {
        auto before = std::prev(after);
        CHECK(before->first + Arena::round(before->second) <= p);
      }
      live[p] = n;
    } else {
      auto it = live.begin();
      std::advance(it, rng() % live.size());
      CHECK(a.release(it->first));
      live.erase(it);
    }
    if (step % 10000 == 0) {
      size_t used = 0;
      for (auto& kv : live) used += Arena::round(kv.second);
      CHECK(used == a.bytesUsed());
    }
  }
  {  // chunks handed back while others hold live ranges: only empty ones go
    auto chunksBefore = a.chunks();
    auto freed = a.takeFreeChunks();
    for (auto& f : freed)
      for (auto& kv : live) CHECK(!(kv.first >= f.first && kv.first < f.first + f.second));
    CHECK(a.chunks().size() + freed.size() == chunksBefore.size());
    for (int t = 0; t < 2000; ++t) {  // later ranges never fall in a returned chunk
      const uint64_t p = a.alloc((size_t)1 << (18 + rng() % 10));
      CHECK(p != 0);
      for (auto& f : freed) CHECK(!(p >= f.first && p < f.first + f.second));
      live[p] = 0;
      CHECK(a.release(p));
      live.erase(p);
    }
  }
  CHECK(!a.release(12345));  // not an address the arena handed out
  for (auto& kv : live) CHECK(a.release(kv.first));
  live.clear();
  CHECK(a.bytesUsed() == 0);
  const size_t nChunks = a.chunks().size();
  CHECK(a.freeRanges() == nChunks);  // every chunk merged back into one range
  auto freed = a.takeFreeChunks();
  CHECK(freed.size() == nChunks && a.chunks().empty());
  {  // growth steps of a fresh arena under small requests, then one larger than a step
    std::vector<size_t> steps;
    uint64_t nb = (uint64_t)1 << 44;
    Arena g([&](size_t bytes) -> uint64_t {
      steps.push_back(bytes);
      const uint64_t base = nb;
      nb += bytes;
      return base;
    });
    const size_t MB = (size_t)1 << 20;
    for (int t = 0; t < 3000; ++t) CHECK(g.alloc(MB) != 0);  // 3000 MB in 1 MB ranges
    const size_t want[] = {64 * MB, 64 * MB, 128 * MB, 256 * MB, 512 * MB, 512 * MB, 512 * MB, 512 * MB, 512 * MB};
    CHECK(steps.size() == sizeof(want) / sizeof(want[0]));
    for (size_t i = 0; i < steps.size() && i < sizeof(want) / sizeof(want[0]); ++i) CHECK(steps[i] == want[i]);
    CHECK(g.alloc(700 * MB) != 0);  // larger than a step: a chunk of its own size
    CHECK(steps.back() == 700 * MB);
  }
  if (fails == 0) std::printf("OK %zu chunks\n", nChunks);
  return fails ? 1 : 0;
}
