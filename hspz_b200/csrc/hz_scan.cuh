// Device-wide exclusive scan (reduce-then-scan, three launches, no
// inter-block waits) and a stable LSD radix sort of (u32 key, u32 value)
// pairs built on it.  Used for seed-count prefixes, stream compaction and
// the on-device seed-table build.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hz {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048

// Sum of one or two u32 streams.
template <typename T> struct Sum;
template <> struct Sum<uint32_t> {
  __device__ __forceinline__ static uint32_t zero() { return 0u; }
  __device__ __forceinline__ static uint32_t add(uint32_t a, uint32_t b) { return a + b; }
  __device__ __forceinline__ static uint32_t shfl_up(uint32_t v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
};
template <> struct Sum<uint2> {
  __device__ __forceinline__ static uint2 zero() { return make_uint2(0u, 0u); }
  __device__ __forceinline__ static uint2 add(uint2 a, uint2 b) { return make_uint2(a.x + b.x, a.y + b.y); }
  __device__ __forceinline__ static uint2 shfl_up(uint2 v, int d) {
    return make_uint2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
  }
};

// A 64-bit hit count paired with a 32-bit position count.
struct HitNz {
  unsigned long long h;
  uint32_t n;
};
template <> struct Sum<HitNz> {
  __device__ __forceinline__ static HitNz zero() { return HitNz{0ull, 0u}; }
  __device__ __forceinline__ static HitNz add(HitNz a, HitNz b) { return HitNz{a.h + b.h, a.n + b.n}; }
  __device__ __forceinline__ static HitNz shfl_up(HitNz v, int d) {
    return HitNz{__shfl_up_sync(0xffffffffu, v.h, d), __shfl_up_sync(0xffffffffu, v.n, d)};
  }
};

// Exclusive block scan of one value per thread; returns the exclusive prefix
// and writes the block total to *total.
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *total) {
  __shared__ T warp_tot[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T up = Sum<T>::shfl_up(incl, d);
    if (lane >= d) incl = Sum<T>::add(incl, up);
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    T w = lane < kScanThreads / 32 ? warp_tot[lane] : Sum<T>::zero();
    T wi = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      T up = Sum<T>::shfl_up(wi, d);
      if (lane >= d) wi = Sum<T>::add(wi, up);
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = wi;  // inclusive warp prefix
  }
  __syncthreads();
  T before = warp == 0 ? Sum<T>::zero() : warp_tot[warp - 1];
  *total = warp_tot[kScanThreads / 32 - 1];
  __syncthreads();
  // exclusive = before + incl - v  (as add of the exclusive lane prefix)
  T lane_excl = Sum<T>::shfl_up(incl, 1);
  if (lane == 0) lane_excl = Sum<T>::zero();
  return Sum<T>::add(before, lane_excl);
}

// Pass 1: per-tile totals.
template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const T *__restrict__ in, uint64_t n,
                                                                   T *__restrict__ partial) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  T acc = Sum<T>::zero();
#pragma unroll
  for (int i = 0; i < kScanItems; i++)
    if (base + i < n) acc = Sum<T>::add(acc, in[base + i]);
  T tot;
  block_exclusive_scan<T>(acc, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// Pass 2: exclusive scan of the tile totals in one block (any count), total
// into *grand.
template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_partials_kernel(T *partial, uint64_t n, T *grand) {
  T carry = Sum<T>::zero();
  for (uint64_t off = 0; off < n; off += kScanTile) {
    uint64_t base = off + (uint64_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T acc = Sum<T>::zero();
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      v[i] = base + i < n ? partial[base + i] : Sum<T>::zero();
      acc = Sum<T>::add(acc, v[i]);
    }
    T tot;
    T ex = Sum<T>::add(carry, block_exclusive_scan<T>(acc, &tot));
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      if (base + i < n) partial[base + i] = ex;
      ex = Sum<T>::add(ex, v[i]);
    }
    carry = Sum<T>::add(carry, tot);
  }
  if (threadIdx.x == 0 && grand) *grand = carry;
}

// Pass 3: per-tile exclusive scan plus the tile offset.
template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const T *__restrict__ in, uint64_t n,
                                                                  const T *__restrict__ partial,
                                                                  T *__restrict__ out) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T acc = Sum<T>::zero();
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    v[i] = base + i < n ? in[base + i] : Sum<T>::zero();
    acc = Sum<T>::add(acc, v[i]);
  }
  T tot;
  T ex = Sum<T>::add(partial[blockIdx.x], block_exclusive_scan<T>(acc, &tot));
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    if (base + i < n) out[base + i] = ex;
    ex = Sum<T>::add(ex, v[i]);
  }
}

inline uint64_t scan_tiles(uint64_t n) { return (n + kScanTile - 1) / kScanTile; }

// Exclusive scan of n elements from `in` to `out` (may alias); `partial`
// needs scan_tiles(n) elements; the grand total lands in *grand (device).
template <typename T>
inline void exclusive_scan(const T *in, T *out, uint64_t n, T *partial, T *grand, cudaStream_t s) {
  uint64_t tiles = scan_tiles(n);
  if (n == 0) {
    cudaMemsetAsync(grand, 0, sizeof(T), s);
    return;
  }
  scan_reduce_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, partial);
  scan_partials_kernel<T><<<1, kScanThreads, 0, s>>>(partial, tiles, grand);
  scan_apply_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, partial, out);
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (key, value) pairs, 8-bit digits.

constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 16;
constexpr int kRadixTile = kRadixThreads * kRadixItems;  // 4096
constexpr int kRadixBins = 256;

// Digit histogram of each tile, stored digit-major: hist[d * tiles + tile].
__global__ void __launch_bounds__(kRadixThreads) radix_hist_kernel(const uint32_t *__restrict__ keys, uint64_t n,
                                                                   int shift, uint32_t *__restrict__ hist,
                                                                   uint64_t tiles) {
  __shared__ uint32_t h[kRadixBins];
  h[threadIdx.x] = 0;
  __syncthreads();
  uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
  for (int i = 0; i < kRadixItems; i++) {
    uint64_t e = base + (uint64_t)i * kRadixThreads + threadIdx.x;
    if (e < n) atomicAdd(&h[(keys[e] >> shift) & 0xFF], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: element order within a tile is round-major, lane-minor,
// and ranks among equal digits follow that order, so the pass is stable.
__global__ void __launch_bounds__(kRadixThreads) radix_scatter_kernel(
    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, uint64_t n, int shift,
    const uint32_t *__restrict__ offsets, uint64_t tiles, uint32_t *__restrict__ keys_out,
    uint32_t *__restrict__ vals_out) {
  constexpr int W = kRadixThreads / 32;
  __shared__ uint32_t base_off[kRadixBins];        // global offset + running tile count
  __shared__ uint32_t warp_cnt[W][kRadixBins];      // per-round per-warp digit counts -> prefixes
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  base_off[threadIdx.x] = offsets[(uint64_t)threadIdx.x * tiles + blockIdx.x];
  uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixItems; r++) {
    for (int w = 0; w < W; w++) warp_cnt[w][threadIdx.x] = 0;
    __syncthreads();
    uint64_t e = base + (uint64_t)r * kRadixThreads + threadIdx.x;
    bool ok = e < n;
    uint32_t k = ok ? keys[e] : 0u;
    uint32_t v = ok ? vals[e] : 0u;
    uint32_t d = ok ? ((k >> shift) & 0xFF) : 0x100u;  // out-of-range lanes form their own group
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t rank = __popc(peers & lanemask_lt());
    if (ok && rank == 0) warp_cnt[warp][d] = __popc(peers);
    __syncthreads();
    {
      // exclusive prefix over warps for digit threadIdx.x
      uint32_t acc = 0;
      for (int w = 0; w < W; w++) {
        uint32_t c = warp_cnt[w][threadIdx.x];
        warp_cnt[w][threadIdx.x] = acc;
        acc += c;
      }
      // stash the round total in a register; apply after the scatter reads base_off
      __syncthreads();
      if (ok) {
        uint32_t dst = base_off[d] + warp_cnt[warp][d] + rank;
        keys_out[dst] = k;
        vals_out[dst] = v;
      }
      __syncthreads();
      base_off[threadIdx.x] += acc;
    }
    __syncthreads();
  }
}

}  // namespace hz
