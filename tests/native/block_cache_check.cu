// Host-only check of the per-context block cache (no CUDA call is made: the
// blocks are fake addresses and flush() is never called).
#include <cstdio>

#include "../../cudanextgenpb_b200/csrc/pbgpu_internal.cuh"

using pbgpu::BlockCache;

static int fails = 0;
#define CHECK(x)                                        \
  do {                                                  \
    if (!(x)) {                                         \
      std::printf("FAIL line %d: %s\n", __LINE__, #x); \
      ++fails;                                          \
    }                                                   \
  } while (0)

static void* addr(size_t i) { return reinterpret_cast<void*>(0x1000 * (i + 1)); }

int main() {
  BlockCache bc;
  size_t got = 0;
  CHECK(bc.take(100, &got) == nullptr);  // empty
  CHECK(bc.put(addr(0), 4096));
  CHECK(bc.put(addr(1), 1 << 20));
  CHECK(bc.put(addr(2), 300000));
  CHECK(bc.bytes == 4096 + (1 << 20) + 300000);
  // smallest block of want .. 2 want + 64 KiB
  CHECK(bc.take(200000, &got) == addr(2) && got == 300000);
  CHECK(bc.take(200000, &got) == nullptr);  // 1 MiB is more than 2 x 200000 + 64 KiB
  CHECK(bc.take(100, &got) == addr(0) && got == 4096);
  CHECK(bc.take(600000, &got) == addr(1) && got == (size_t(1) << 20));
  CHECK(bc.blks.empty() && bc.bytes == 0);
  // byte cap
  CHECK(bc.put(addr(3), BlockCache::kMaxBytes));
  CHECK(!bc.put(addr(4), 1));
  CHECK(bc.take(BlockCache::kMaxBytes, &got) == addr(3));
  // block cap
  for (size_t i = 0; i < BlockCache::kMaxBlocks; ++i) CHECK(bc.put(addr(10 + i), 256));
  CHECK(!bc.put(addr(9999), 256));
  CHECK(bc.blks.size() == BlockCache::kMaxBlocks && bc.bytes == 256 * BlockCache::kMaxBlocks);
  if (fails == 0) std::printf("block cache ok\n");
  return fails == 0 ? 0 : 1;
}
