// radix_sort.cuh -- stable LSD radix sort of (uint32 cell key, int32 index)
// pairs, the B200 replacement of thrust::stable_sort_by_key in the reference
// (Collision_Detection_BroadPhase.cuh:110-117).  Stability makes the result
// unique, so the permutation equals the reference's bit for bit.
//
// Only the significant key bits are sorted (cell keys need ~20 of 32).  Per
// pass of kRadixBits bits, three kernels:
//   1. histogram: per tile of kTileKeys keys, digit counts -> counts[digit][tile]
//   2. scan:      one block per digit scans its row across tiles (exclusive)
//                 and emits the digit total
//   3. scatter:   each tile ranks its keys stably (warp match + per-warp
//                 digit counters in shared memory, warps in key order) and
//                 writes key/index to digit base + tile offset + local rank.
// Keys are read twice and written once per pass; indices read and written
// once (the first pass generates them).  Traffic ~ 20 B/key/pass.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace blaze {

constexpr int kRadixBits = 8;
constexpr int kRadixDigits = 1 << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;
constexpr int kTileKeys = kSortThreads * kSortItems;

struct RadixSortBuffers {
  uint32_t* keys[2];
  int32_t* vals[2];
  uint32_t* counts;   // kRadixDigits * max_tiles
  uint32_t* totals;   // kRadixDigits
  int max_n;
  int max_tiles;
};

// Bytes of device scratch the sort needs for n keys (besides keys/vals).
size_t radix_scratch_bytes(int n);

// Sort keys[0]/vals (vals generated as 0..n-1 when gen_vals) over the low
// `bits` bits.  Result lands in keys[res]/vals[res]; returns res.
// `gate` (may be null): when non-null and *gate == 0 every kernel returns at
// once, so the launch sequence can stay fixed while the work is skipped.
int radix_sort_pairs(RadixSortBuffers& b, int n, int bits, bool gen_vals, const int* gate,
                     cudaStream_t stream);

}  // namespace blaze
