// radix_sort.cu -- see radix_sort.cuh.
#include "radix_sort.cuh"

namespace blaze {

namespace {

__device__ __forceinline__ bool gated_off(const int* gate) { return gate != nullptr && *gate == 0; }

__global__ void __launch_bounds__(kSortThreads)
k_radix_hist(const uint32_t* __restrict__ keys, int n, int shift, int tiles,
             uint32_t* __restrict__ counts, const int* gate) {
  if (gated_off(gate)) return;
  __shared__ uint32_t cnt[kRadixDigits];
  for (int d = threadIdx.x; d < kRadixDigits; d += kSortThreads) cnt[d] = 0;
  __syncthreads();
  const int base = blockIdx.x * kTileKeys;
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    int i = base + k * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&cnt[(__ldg(keys + i) >> shift) & (kRadixDigits - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadixDigits; d += kSortThreads)
    counts[(size_t)d * tiles + blockIdx.x] = cnt[d];
}

// One block per digit: exclusive scan of that digit's per-tile counts.
__global__ void __launch_bounds__(kSortThreads)
k_radix_scan(uint32_t* __restrict__ counts, int tiles, uint32_t* __restrict__ totals,
             const int* gate) {
  if (gated_off(gate)) return;
  __shared__ uint32_t warp_sum[kSortWarps];
  uint32_t* row = counts + (size_t)blockIdx.x * tiles;
  const int per = (tiles + kSortThreads - 1) / kSortThreads;
  const int b0 = threadIdx.x * per;
  uint32_t s = 0;
  for (int k = 0; k < per; ++k)
    if (b0 + k < tiles) s += row[b0 + k];
  // block exclusive scan of s
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sum[w] = x;
  __syncthreads();
  uint32_t woff = 0, total = 0;
#pragma unroll
  for (int q = 0; q < kSortWarps; ++q) {
    uint32_t v = warp_sum[q];
    if (q < w) woff += v;
    total += v;
  }
  uint32_t run = woff + x - s;  // exclusive prefix of this thread's chunk
  for (int k = 0; k < per; ++k) {
    if (b0 + k < tiles) {
      uint32_t c = row[b0 + k];
      row[b0 + k] = run;
      run += c;
    }
  }
  if (threadIdx.x == 0) totals[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kSortThreads)
k_radix_scatter(const uint32_t* __restrict__ keys_in, const int32_t* __restrict__ vals_in,
                uint32_t* __restrict__ keys_out, int32_t* __restrict__ vals_out, int n, int shift,
                int tiles, const uint32_t* __restrict__ counts, const uint32_t* __restrict__ totals,
                bool gen_vals, const int* gate) {
  if (gated_off(gate)) return;
  __shared__ uint32_t base_s[kRadixDigits];
  __shared__ uint32_t wcnt[kSortWarps][kRadixDigits];
  __shared__ uint32_t wsum[kSortWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

  // digit bases: exclusive scan of totals + this tile's offset in each digit
  {
    const int d = threadIdx.x;  // kSortThreads == kRadixDigits
    uint32_t t = totals[d];
    uint32_t x = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    for (int q = 0; q < kSortWarps; ++q) wcnt[q][d] = 0;
    __syncthreads();
    uint32_t off = 0;
    for (int q = 0; q < w; ++q) off += wsum[q];
    base_s[d] = off + x - t + counts[(size_t)d * tiles + blockIdx.x];
  }
  __syncthreads();

  const unsigned lt = (1u << lane) - 1u;
  const int tbase = blockIdx.x * kTileKeys + w * (32 * kSortItems);
  uint32_t key[kSortItems];
  int32_t val[kSortItems];
  uint32_t rank[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const int i = tbase + k * 32 + lane;
    const bool valid = i < n;
    key[k] = valid ? __ldg(keys_in + i) : 0u;
    val[k] = valid ? (gen_vals ? i : __ldg(vals_in + i)) : 0;
    const uint32_t d = valid ? ((key[k] >> shift) & (kRadixDigits - 1)) : (uint32_t)kRadixDigits;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t b = 0;
    if (valid) b = wcnt[w][d];
    __syncwarp();
    if (valid && lane == leader) wcnt[w][d] = b + __popc(peers);
    __syncwarp();
    rank[k] = b + __popc(peers & lt);
  }
  __syncthreads();
  // per-digit exclusive offsets across warps (warps hold consecutive keys)
  {
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int q = 0; q < kSortWarps; ++q) {
      uint32_t c = wcnt[q][d];
      wcnt[q][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const int i = tbase + k * 32 + lane;
    if (i < n) {
      const uint32_t d = (key[k] >> shift) & (kRadixDigits - 1);
      const uint32_t pos = base_s[d] + wcnt[w][d] + rank[k];
      keys_out[pos] = key[k];
      vals_out[pos] = val[k];
    }
  }
}

}  // namespace

size_t radix_scratch_bytes(int n) {
  int tiles = (n + kTileKeys - 1) / kTileKeys;
  return sizeof(uint32_t) * ((size_t)kRadixDigits * (tiles > 0 ? tiles : 1) + kRadixDigits);
}

int radix_sort_pairs(RadixSortBuffers& b, int n, int bits, bool gen_vals, const int* gate,
                     cudaStream_t stream) {
  static_assert(kSortThreads == kRadixDigits, "one thread per digit in the scatter prologue");
  const int tiles = (n + kTileKeys - 1) / kTileKeys;
  if (n <= 0) return 0;
  int passes = (bits + kRadixBits - 1) / kRadixBits;
  if (passes < 1) passes = 1;
  int cur = 0;
  for (int p = 0; p < passes; ++p) {
    const int shift = p * kRadixBits;
    k_radix_hist<<<tiles, kSortThreads, 0, stream>>>(b.keys[cur], n, shift, tiles, b.counts, gate);
    k_radix_scan<<<kRadixDigits, kSortThreads, 0, stream>>>(b.counts, tiles, b.totals, gate);
    k_radix_scatter<<<tiles, kSortThreads, 0, stream>>>(b.keys[cur], b.vals[cur], b.keys[cur ^ 1],
                                                         b.vals[cur ^ 1], n, shift, tiles, b.counts,
                                                         b.totals, gen_vals && p == 0, gate);
    cur ^= 1;
  }
  return cur;
}

}  // namespace blaze
