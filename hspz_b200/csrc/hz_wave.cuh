// The wave pipeline: any number of seed_and_filter calls (one WGA chunk of
// one strand of one query each) processed by one fixed sequence of launches.
//
//   lookup_count   per query position: the capped hit counts of its seeds
//   np_*           scan of the counts; compaction of positions with hits
//   scopes         per call: hit range and MAX_HITS dedup scopes
//   gate           fused hit expansion + thread-per-hit X-drop score gate
//   long           lane-per-candidate exact extension of the gate's long candidates
//   exact          warp-per-candidate X-drop positions, entropy, accept
//
// Semantics follow hspZ src/gpu/kernels.rs and src/gpu/mod.rs (cited per
// kernel).  Hit indices are 64-bit across a wave (a call's own hit count is
// a u32, as in the reference).  Sizes that depend on the data (hits,
// candidates, HSPs) are read from device memory, so a wave needs no host
// round trip until its output.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "hz_device.cuh"
#include "hz_scan.cuh"

namespace hz {

// One seed_and_filter call of a wave.
struct CallDev {
  uint32_t qoff;     // offset of the strand block's position 0 in the query store
  uint32_t qlen;     // block length (right edge of the extension)
  uint32_t start;    // first seed position of the call (block coordinates)
  uint32_t pos_off;  // first flat position of the call in the wave
};

// Inputs shared by the lookup, scope and gate kernels.
struct WaveIn {
  const uint8_t *ref;  // reference codes (padded on both sides)
  uint32_t rlen;
  const uint8_t *qbuf;  // query store (padded)
  const uint32_t *index_table;
  const uint32_t *pos_table;
  const CallDev *calls;
  uint32_t ncalls;
  uint32_t npos;          // flat positions of the wave
  const uint64_t *seeds;  // host-uploaded seeds (one per flat position) or null
  ShapeDev shape;
  uint32_t per_pos;  // seeds per position: 1 + kmer_size with transitions, else 1
  uint32_t occ_cap;
  const uint32_t *nbr_hits;  // per k-mer hits of all 1 + kmer_size seeds, or null
  // the query store packed 2 bits per base (forward half of pack2_kernel's
  // records), or null to read the 8-bit codes
  const uint4 *qp2;
  uint32_t *pos_kmer;  // per flat position: its k-mer, written by lookup_count (or null)
};

// Device-side counters of a wave.
struct WaveTotals {
  unsigned long long hits;   // seed hits of the wave
  unsigned long long cells;  // scalar X-drop cells scored
  unsigned long long valid;  // valid seed windows
  unsigned long long tiles;  // gate work-queue cursor
  uint32_t nz;               // positions with at least one hit
  uint32_t n_scopes;
  uint32_t status;  // bit 0: a call's first seed alone exceeds max_hits; bit 1: a call exceeds 2^32 hits
  uint32_t cand;    // gate candidates written (may exceed capacity)
  uint32_t raw;     // accepted HSPs written (may exceed capacity)
  uint32_t long_next;  // long_kernel's cursor over the candidates
  uint32_t pad[2];
};

// Gate candidate: a hit whose score bound passes the threshold, or whose
// extension ran past the per-direction cap ("long").
struct Cand {
  uint32_t scope;  // dedup scope of the hit
  uint32_t r0;     // reference anchor
  uint32_t q0;     // query anchor, absolute in the query store
  uint32_t call;   // call index | kLongFlag | kDoneFlag
  int32_t rmax;    // the right and left maxima: the gate's, or long_kernel's (kDoneFlag)
  int32_t lmax;
  int32_t rpos;    // their positions, filled in by long_kernel only
  int32_t lpos;
};
constexpr uint32_t kLongFlag = 1u << 31;

__device__ __forceinline__ uint32_t call_of(const CallDev *calls, uint32_t ncalls, uint32_t p) {
  uint32_t lo = 0, hi = ncalls;  // last call with pos_off <= p
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (calls[mid].pos_off <= p) lo = mid; else hi = mid;
  }
  return lo;
}

// Seed of flat position p: (query position, k-mer); false for an invalid
// window.  src/seed.rs:88-123.
__device__ __forceinline__ bool position_seed(const WaveIn &w, const CallDev &c, uint32_t p, uint32_t *qpos,
                                              uint32_t *kmer) {
  if (w.seeds) {
    uint64_t s = w.seeds[p];
    *kmer = (uint32_t)(s >> 32);
    *qpos = (uint32_t)s;
    return true;
  }
  *qpos = c.start + (p - c.pos_off);
  *kmer = w.qp2 ? kmer_packed(w.qp2, c.qoff + *qpos, w.shape) : kmer_at(w.qbuf + c.qoff, *qpos, w.shape);
  return *kmer != kInvalidKmer;
}

// Seed v of a position: the exact k-mer, then kmer ^ (2 << 2(v-1))
// (push_seeds, src/seed.rs:107-123).
__device__ __forceinline__ uint32_t seed_variant(uint32_t kmer, uint32_t v) {
  return v == 0 ? kmer : kmer ^ (2u << (2 * (v - 1)));
}

// find_num_hits with the occurrence cap (src/gpu/kernels.rs:70-115).
__device__ __forceinline__ uint32_t bucket(const WaveIn &w, uint32_t k, uint32_t *beg) {
  uint32_t end = __ldg(w.index_table + k);
  uint32_t b = k ? __ldg(w.index_table + k - 1) : 0u;
  uint32_t c = end - b;
  if (w.occ_cap && c > w.occ_cap) c = 0;
  *beg = b;
  return c;
}

// Per k-mer: the capped hit counts of its exact seed and of its kmer_size
// transition seeds, summed -- what lookup_count adds up for a query
// position with that k-mer (u32, wrapping like that sum).
__global__ void nbr_hits_kernel(const uint32_t *__restrict__ index_table, uint64_t n, uint32_t kmer_size,
                                uint32_t occ_cap, uint32_t *__restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t kmer = (uint32_t)i;
    uint32_t hi[kMaxCare + 1], lo[kMaxCare + 1];
#pragma unroll
    for (uint32_t v = 0; v < kMaxCare + 1; v++) {
      hi[v] = lo[v] = 0;
      if (v <= kmer_size) {
        const uint32_t k = seed_variant(kmer, v);
        hi[v] = __ldg(index_table + k);
        lo[v] = k ? __ldg(index_table + k - 1) : 0u;
      }
    }
    uint32_t sum = 0;
#pragma unroll
    for (uint32_t v = 0; v < kMaxCare + 1; v++) {
      uint32_t c = hi[v] - lo[v];
      if (occ_cap && c > occ_cap) c = 0;
      sum += c;
    }
    out[i] = sum;
  }
}

// last index in [lo, hi) whose value is <= h (caller guarantees one exists)
__device__ __forceinline__ uint32_t last_le(const unsigned long long *v, uint32_t lo, uint32_t hi,
                                            unsigned long long h) {
  uint32_t a = lo, b = hi;  // first index with v > h
  while (a < b) {
    uint32_t m = (a + b) >> 1;
    if (v[m] <= h) a = m + 1; else b = m;
  }
  return a - 1;
}

// ---------------------------------------------------------------------------
// Per flat position: total hits of its seeds.  A block walks `chunks`
// consecutive chunks of kCountPerBlock positions (up to 16, fewer when the
// wave is small, so that every SM still gets blocks), so the search for its
// first call (log2(calls) dependent loads) is paid once per block and the
// threads' calls only advance after it.  With the neighbourhood table and
// the packed query, a thread takes four consecutive positions of a chunk:
// one 32-base window gives their four k-mers, their four counts are
// gathered together, and counts and k-mers go out as 16-byte stores.
constexpr int kCountThreads = 256;
constexpr int kCountPerBlock = 1024;
constexpr uint32_t kCountMaxChunks = 16;

// Chunks per block for a wave of npos positions: as many as keep at least
// ~600 blocks (four per SM) in the grid.
inline uint32_t lookup_chunks(uint64_t npos) {
  const uint64_t per = npos / (600ull * kCountPerBlock);
  return (uint32_t)(per < 1 ? 1 : per > kCountMaxChunks ? kCountMaxChunks : per);
}

__global__ void __launch_bounds__(kCountThreads) lookup_count_kernel(WaveIn w, uint32_t chunks,
                                                                     uint32_t *__restrict__ pos_hits,
                                                                     WaveTotals *__restrict__ tot) {
  __shared__ uint32_t s_c0;
  const uint32_t base = blockIdx.x * chunks * kCountPerBlock;
  if (threadIdx.x == 0) s_c0 = call_of(w.calls, w.ncalls, base);
  __syncthreads();
  uint32_t c = s_c0;
  uint32_t valid = 0;
  constexpr int kPer = kCountPerBlock / kCountThreads;
  static_assert(kPer % 4 == 0, "a thread's counts go out as 16-byte stores");
  const bool by_table = w.nbr_hits && w.per_pos > 1;
  // kPer consecutive positions per thread from one 32-base packed window
  const bool by_window = by_table && w.qp2 && !w.seeds && w.shape.size + kPer - 1 <= 32;
  const uint32_t win_mask = w.shape.size >= 32 ? 0xFFFFFFFFu : (1u << w.shape.size) - 1u;
#pragma unroll 1
  for (uint32_t chunk = 0; chunk < chunks; chunk++) {
    const uint32_t p0 = base + chunk * kCountPerBlock;
    if (p0 >= w.npos) break;
    if (by_window) {
      const uint32_t p = p0 + kPer * threadIdx.x;
      if (p >= w.npos) continue;
      while (c + 1 < w.ncalls && w.calls[c + 1].pos_off <= p) c++;
      const CallDev cd = w.calls[c];
      const uint32_t next_off = c + 1 < w.ncalls ? w.calls[c + 1].pos_off : 0xFFFFFFFFu;
      uint32_t kmer[kPer], sum[kPer];
      if (p + kPer - 1 < next_off && p + kPer - 1 < w.npos) {  // positions of one call: one window
        uint32_t lo, hi, sp;
        window32(w.qp2, cd.qoff + cd.start + (p - cd.pos_off), &lo, &hi, &sp);
        const uint64_t w64 = (uint64_t)hi << 32 | lo;
#pragma unroll
        for (uint32_t j = 0; j < kPer; j++)
          kmer[j] = ((sp >> j) & win_mask) ? kInvalidKmer
                    : w.shape.is_12of19          ? kmer_12of19(lo, hi, j)
                                                 : kmer_runs(w64, j, w.shape);
      } else {  // a call boundary or the wave's end among them
        uint32_t cc = c;
#pragma unroll
        for (uint32_t j = 0; j < kPer; j++) {
          kmer[j] = kInvalidKmer;
          if (p + j < w.npos) {
            while (cc + 1 < w.ncalls && w.calls[cc + 1].pos_off <= p + j) cc++;
            uint32_t qpos;
            position_seed(w, w.calls[cc], p + j, &qpos, &kmer[j]);
          }
        }
      }
#pragma unroll
      for (uint32_t j = 0; j < kPer; j++) {
        sum[j] = 0;
        if (kmer[j] != kInvalidKmer) {
          valid++;
          sum[j] = __ldg(w.nbr_hits + kmer[j]);
        }
      }
      if (p + kPer - 1 < w.npos) {
#pragma unroll
        for (uint32_t j = 0; j < kPer; j += 4) {
          *reinterpret_cast<uint4 *>(pos_hits + p + j) = make_uint4(sum[j], sum[j + 1], sum[j + 2], sum[j + 3]);
          if (w.pos_kmer)
            *reinterpret_cast<uint4 *>(w.pos_kmer + p + j) =
                make_uint4(kmer[j], kmer[j + 1], kmer[j + 2], kmer[j + 3]);
        }
      } else {
#pragma unroll
        for (uint32_t j = 0; j < kPer; j++)
          if (p + j < w.npos) {
            pos_hits[p + j] = sum[j];
            if (w.pos_kmer) w.pos_kmer[p + j] = kmer[j];
          }
      }
      continue;
    }
    if (by_table) {
      // all of the thread's k-mers first, then their neighbourhood counts, so
      // the count gathers of its positions are in flight together
      uint32_t kmer[kPer];
#pragma unroll
      for (int i = 0; i < kPer; i++) {
        const uint32_t p = p0 + i * kCountThreads + threadIdx.x;
        kmer[i] = kInvalidKmer;
        if (p < w.npos) {
          while (c + 1 < w.ncalls && w.calls[c + 1].pos_off <= p) c++;
          uint32_t qpos;
          position_seed(w, w.calls[c], p, &qpos, &kmer[i]);
        }
      }
      uint32_t sum[kPer];
#pragma unroll
      for (int i = 0; i < kPer; i++) {
        sum[i] = 0;
        if (kmer[i] != kInvalidKmer) {
          valid++;
          sum[i] = __ldg(w.nbr_hits + kmer[i]);
        }
      }
#pragma unroll
      for (int i = 0; i < kPer; i++) {
        const uint32_t p = p0 + i * kCountThreads + threadIdx.x;
        if (p < w.npos) {
          pos_hits[p] = sum[i];
          if (w.pos_kmer) w.pos_kmer[p] = kmer[i];
        }
      }
      continue;
    }
#pragma unroll 1
    for (int i = 0; i < kPer; i++) {
      uint32_t p = p0 + i * kCountThreads + threadIdx.x;
      if (p >= w.npos) break;
      while (c + 1 < w.ncalls && w.calls[c + 1].pos_off <= p) c++;
      CallDev cd = w.calls[c];
      uint32_t qpos, kmer, sum = 0;
      if (position_seed(w, cd, p, &qpos, &kmer)) {
        valid++;
        // every seed's bucket bounds are loaded before any is used, so the
        // loads are in flight together
        uint32_t hi[kMaxCare + 1], lo[kMaxCare + 1];
#pragma unroll
        for (uint32_t v = 0; v < kMaxCare + 1; v++) {
          hi[v] = lo[v] = 0;
          if (v < w.per_pos) {
            const uint32_t k = seed_variant(kmer, v);
            hi[v] = __ldg(w.index_table + k);
            lo[v] = k ? __ldg(w.index_table + k - 1) : 0u;
          }
        }
#pragma unroll
        for (uint32_t v = 0; v < kMaxCare + 1; v++) {
          uint32_t cnt = hi[v] - lo[v];
          if (w.occ_cap && cnt > w.occ_cap) cnt = 0;  // find_num_hits with the occurrence cap
          sum += cnt;
        }
      }
      pos_hits[p] = sum;
      if (w.pos_kmer) w.pos_kmer[p] = kmer;
    }
  }
  for (int d = 16; d > 0; d >>= 1) valid += __shfl_down_sync(0xffffffffu, valid, d);
  if ((threadIdx.x & 31) == 0 && valid) atomicAdd(&tot->valid, (unsigned long long)valid);
}

// Scan of (hits, has-hits) over positions, then compaction of the positions
// with hits: np_excl = hits of the wave before the position, np_pos = its
// flat index, np_kmer = its k-mer (when lookup_count kept the k-mers).
__global__ void __launch_bounds__(kScanThreads) np_reduce_kernel(const uint32_t *__restrict__ pos_hits, uint64_t n,
                                                                 HitNz *__restrict__ partial) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  HitNz acc = HitNz{0ull, 0u};
#pragma unroll
  for (int i = 0; i < kScanItems; i++)
    if (base + i < n) {
      uint32_t h = pos_hits[base + i];
      acc.h += h;
      acc.n += h > 0;
    }
  HitNz tot;
  block_exclusive_scan<HitNz>(acc, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) np_emit_kernel(const uint32_t *__restrict__ pos_hits, uint64_t n,
                                                               const HitNz *__restrict__ partial,
                                                               unsigned long long *__restrict__ np_excl,
                                                               uint32_t *__restrict__ np_pos,
                                                               const uint32_t *__restrict__ pos_kmer,
                                                               uint32_t *__restrict__ np_kmer) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  HitNz acc = HitNz{0ull, 0u};
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    v[i] = base + i < n ? pos_hits[base + i] : 0u;
    acc.h += v[i];
    acc.n += v[i] > 0;
  }
  // the k-mers of the positions with hits, loaded while the block scans
  uint32_t km[kScanItems];
#pragma unroll
  for (int i = 0; i < kScanItems; i++) km[i] = np_kmer && v[i] ? pos_kmer[base + i] : 0u;
  HitNz tot;
  HitNz ex = block_exclusive_scan<HitNz>(acc, &tot);
  HitNz off = partial[blockIdx.x];
  ex.h += off.h;
  ex.n += off.n;
#pragma unroll
  for (int i = 0; i < kScanItems; i++) {
    if (v[i]) {
      np_excl[ex.n] = ex.h;
      np_pos[ex.n] = (uint32_t)(base + i);
      if (np_kmer) np_kmer[ex.n] = km[i];
      ex.h += v[i];
      ex.n += 1;
    }
  }
}

// The gate's tile table: tile_first[j] = the position with hits that holds
// wave hit j * tile (positions tile the hit space, so every tile start has
// exactly one), tile_call[j] = the call of that position, and
// tile_first[n_tiles] = nz.  Lets a gate warp find its positions and call
// with three loads instead of searches.  Sets status bit 2 when the
// table is too small (the wave is then rerun with a larger one).
__global__ void tile_table_kernel(const unsigned long long *__restrict__ np_excl, const uint32_t *__restrict__ pos_hits,
                                  const uint32_t *__restrict__ np_pos, const CallDev *__restrict__ calls,
                                  uint32_t ncalls, WaveTotals *__restrict__ t, uint32_t tile,
                                  uint32_t *__restrict__ tile_first, uint32_t *__restrict__ tile_call, uint32_t cap) {
  const uint32_t nz = t->nz;
  const unsigned long long total = t->hits;
  const unsigned long long n_tiles = (total + tile - 1) / tile;
  if (n_tiles + 1 > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&t->status, 4u);
    return;
  }
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nz; k += stride) {
    const uint32_t p = np_pos[k];
    unsigned long long lo = np_excl[k], hi = lo + pos_hits[p];
    unsigned long long j = (lo + tile - 1) / tile;
    if (j * tile >= hi) continue;
    const uint32_t c = call_of(calls, ncalls, p);
    for (; j * tile < hi; j++) {
      tile_first[j] = k;
      tile_call[j] = c;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) tile_first[n_tiles] = nz;
}

// Grand totals of the scan into WaveTotals, and the sentinel np_excl[nz].
__global__ void np_totals_kernel(const HitNz *__restrict__ grand, WaveTotals *__restrict__ t,
                                 unsigned long long *__restrict__ np_excl) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    t->hits = grand->h;
    t->nz = grand->n;
    np_excl[grand->n] = grand->h;
  }
}

// ---------------------------------------------------------------------------
// Per call: hit range, and the MAX_HITS dedup scopes (chunk_limits,
// src/gpu/mod.rs:2394-2420, and the single-chunk shortcut when num_hits <=
// max_hits, :1693-1705).  One block; calls are processed in rounds of
// blockDim with a running scope offset, so scopes come out in call order and
// tile the wave's hit space: scope s is [scope_lo[s], scope_lo[s+1]).  A cut
// is the largest cumulative seed hit count below the running limit; it is
// found over the positions with hits and refined by recounting the seeds of
// the position the cut falls in (positions without hits repeat the
// cumulative value before them, so they never move a cut).
constexpr int kScopeThreads = 1024;

__global__ void __launch_bounds__(kScopeThreads) scopes_kernel(WaveIn w, const unsigned long long *__restrict__ np_excl,
                                                               const uint32_t *__restrict__ np_pos,
                                                               WaveTotals *__restrict__ tot, uint32_t max_hits,
                                                               unsigned long long *__restrict__ call_hit_lo,
                                                               uint32_t *__restrict__ call_nz_lo,
                                                               unsigned long long *__restrict__ scope_lo,
                                                               uint32_t *__restrict__ scope_call, uint32_t scope_cap) {
  __shared__ uint32_t s_w[32];
  __shared__ uint32_t s_carry;
  const unsigned long long total = tot->hits;
  const uint32_t nz = tot->nz;
  for (uint32_t c = threadIdx.x; c <= w.ncalls; c += blockDim.x) {
    uint32_t k = nz;
    if (c < w.ncalls) {
      uint32_t p = w.calls[c].pos_off;
      uint32_t a = 0, b = nz;  // first position with hits at or after the call start
      while (a < b) {
        uint32_t m = (a + b) >> 1;
        if (np_pos[m] < p) a = m + 1; else b = m;
      }
      k = a;
    }
    call_nz_lo[c] = k;
    call_hit_lo[c] = k < nz ? np_excl[k] : total;
  }
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint32_t r0 = 0; r0 < w.ncalls; r0 += blockDim.x) {
    uint32_t c = r0 + threadIdx.x;
    uint32_t nsc = 0;
    unsigned long long lo = 0, nh = 0;
    if (c < w.ncalls) {
      lo = call_hit_lo[c];
      nh = call_hit_lo[c + 1] - lo;
      if (nh > 0xFFFFFFFFull) {
        atomicOr(&tot->status, 2u);
        nh = 0;
      }
      nsc = nh <= max_hits ? 1u : (uint32_t)(nh / max_hits) + 1u;
    }
    uint32_t incl = nsc;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t up = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += up;
    }
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      uint32_t xi = s_w[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        uint32_t up = __shfl_up_sync(0xffffffffu, xi, d);
        if (lane >= d) xi += up;
      }
      s_w[lane] = xi;
    }
    __syncthreads();
    uint32_t s0 = s_carry + (wid ? s_w[wid - 1] : 0u) + incl - nsc;
    uint32_t round_total = s_w[31];
    if (c < w.ncalls && s0 + nsc <= scope_cap) {
      scope_lo[s0] = lo;
      scope_call[s0] = c;
      if (nsc > 1) {
        // the first real seed: the reference's walk has no cut when it
        // alone holds >= max_hits hits (lower_bound - 1 underflows)
        CallDev cd = w.calls[c];
        uint32_t span = c + 1 < w.ncalls ? w.calls[c + 1].pos_off - cd.pos_off : w.npos - cd.pos_off;
        for (uint32_t i = 0; i < span; i++) {
          uint32_t qpos, kmer;
          if (position_seed(w, cd, cd.pos_off + i, &qpos, &kmer)) {
            uint32_t beg;
            if (bucket(w, kmer, &beg) >= max_hits) atomicOr(&tot->status, 1u);
            break;
          }
        }
        uint32_t klo = call_nz_lo[c], khi = call_nz_lo[c + 1];
        uint32_t limit = max_hits;  // relative to lo
        for (uint32_t it = 1; it < nsc; it++) {
          // last position of the call whose first hit is below the limit
          uint32_t a = klo, b = khi;
          while (a < b) {
            uint32_t m = (a + b) >> 1;
            if (np_excl[m] - lo < limit) a = m + 1; else b = m;
          }
          uint32_t B = 0;
          if (a > klo) {
            uint32_t k = a - 1;
            uint32_t e = (uint32_t)(np_excl[k] - lo);
            B = e;
            uint32_t p = np_pos[k];
            CallDev pc = w.calls[call_of(w.calls, w.ncalls, p)];
            uint32_t qpos, kmer;
            position_seed(w, pc, p, &qpos, &kmer);
            uint32_t run = e;
            for (uint32_t v = 0; v < w.per_pos; v++) {
              uint32_t beg;
              run += bucket(w, seed_variant(kmer, v), &beg);
              if (run < limit) B = run; else break;
            }
          }
          scope_lo[s0 + it] = lo + B;
          scope_call[s0 + it] = c;
          limit = B + max_hits;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) s_carry += round_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    tot->n_scopes = s_carry;
    if (s_carry < scope_cap) scope_lo[s_carry] = total;
  }
}

}  // namespace hz

#include "hz_gate.cuh"
#include "hz_gate2.cuh"
#include "hz_long.cuh"

namespace hz {

// ---------------------------------------------------------------------------
// Exact extension, one warp per candidate (find_hsps, src/gpu/kernels.rs:
// 1279-1543): the positions of both maxima -- from the gate's maxima with one
// sum scan per 32 cells, or, for a long candidate, the whole extension with
// sum and maximum scans -- then the entropy correction and the final
// threshold (:1555-1701).

struct ExactArgs {
  const uint8_t *ref;
  uint32_t rlen;
  const uint8_t *qbuf;
  const CallDev *calls;
  const Cand *cand;
  uint32_t cand_cap;
  WaveTotals *tot;
  int32_t sub[64];
  int32_t xdrop;
  int32_t hspthresh;
  uint32_t noentropy;
  SegmentPair *raw;
  uint32_t *raw_scope;
  uint32_t raw_cap;
};

__device__ __forceinline__ int32_t warp_incl_sum(int32_t v, uint32_t lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int32_t up = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= (uint32_t)d) v = (int32_t)((uint32_t)v + (uint32_t)up);
  }
  return v;
}

// shuffle-up hands lanes below the offset their own value, so max(v, v) is a no-op
__device__ __forceinline__ int32_t warp_incl_max(int32_t v) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int32_t up = __shfl_up_sync(0xffffffffu, v, d);
    if (up >= v) v = up;
  }
  return v;
}

// One direction of a long candidate, four consecutive cells per lane, 128
// cells per warp step: the lane sums its four cells, the warp scans the lane
// totals and the lanes' largest sums; the first dropping cell (ballot), the
// maximum before it and that maximum's earliest position (ballot of the lanes
// holding it) follow; returns (max, position) and adds the scored cells.
template <bool LEFT>
__device__ __forceinline__ void exact_dir4(const uint8_t *ref, const uint8_t *qry, const int32_t *sub, int32_t X,
                                           uint32_t r0, uint32_t q0, uint32_t nmax, uint32_t lane, int32_t *out_max,
                                           int32_t *out_pos, unsigned long long *cells) {
  int32_t prev_s = 0, prev_m = 0, prev_pos = LEFT ? 0 : -1;
  for (uint32_t tile = 0;; tile += 128) {
    const uint32_t k0 = tile + 4u * lane;
    int32_t p[4];
    int32_t acc = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const uint32_t k = k0 + (uint32_t)i;
      int32_t sc = 0;
      if (k < nmax) {
        uint32_t rc = LEFT ? ref[r0 - 1 - k] : ref[r0 + k];
        uint32_t qc = LEFT ? qry[q0 - 1 - k] : qry[q0 + k];
        sc = sub[rc * kNuc + qc];
      }
      acc = (int32_t)((uint32_t)acc + (uint32_t)sc);
      p[i] = acc;
    }
    const int32_t incl = warp_incl_sum(acc, lane);
    const int32_t base = (int32_t)((uint32_t)prev_s + (uint32_t)incl - (uint32_t)acc);
    int32_t ts[4], lm[4];  // running sums of the lane's cells; the lane's running maximum of them
#pragma unroll
    for (int i = 0; i < 4; i++) {
      ts[i] = (int32_t)((uint32_t)base + (uint32_t)p[i]);
      lm[i] = i ? max(lm[i - 1], ts[i]) : ts[i];
    }
    // the running maximum before the lane's first cell: prev_m and every
    // earlier lane's cells
    const int32_t upto = warp_incl_max(max(lm[3], prev_m));
    int32_t before = __shfl_up_sync(0xffffffffu, upto, 1);
    if (lane == 0) before = prev_m;
    int32_t Mi[4];
    uint32_t dbits = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      Mi[i] = max(before, lm[i]);
      dbits |= (uint32_t)((int32_t)((uint32_t)Mi[i] - (uint32_t)ts[i]) > X) << i;
    }
    const uint32_t dl = __ballot_sync(0xffffffffu, dbits != 0);
    uint32_t first = 128;
    if (dl) {
      const uint32_t fl = (uint32_t)(__ffs(dl) - 1);
      const uint32_t fi = (uint32_t)(__ffs(__shfl_sync(0xffffffffu, dbits, fl)) - 1);
      first = 4u * fl + fi;
    }
    // the maximum before the first dropping cell (or over the whole step)
    int32_t mx;
    if (first == 0) {
      mx = prev_m;
    } else {
      const uint32_t c = first - 1, src = c >> 2, idx = c & 3u;
      int32_t mine = Mi[0];
#pragma unroll
      for (int i = 1; i < 4; i++)
        if ((uint32_t)i == idx) mine = Mi[i];
      mx = __shfl_sync(0xffffffffu, mine, src);
    }
    int32_t pos;
    if (mx == prev_m) {
      pos = prev_pos;
    } else {
      uint32_t wbits = 0;
#pragma unroll
      for (int i = 0; i < 4; i++) wbits |= (uint32_t)(ts[i] == mx && 4u * lane + (uint32_t)i < first) << i;
      const uint32_t wl = __ballot_sync(0xffffffffu, wbits != 0);
      const uint32_t l = (uint32_t)(__ffs(wl) - 1);
      const uint32_t wi = (uint32_t)(__ffs(__shfl_sync(0xffffffffu, wbits, l)) - 1);
      pos = (int32_t)(4u * l + wi + tile) + (LEFT ? 1 : 0);
    }
    if (dl) {
      *cells += min(tile + first + 1, nmax);
      *out_max = mx;
      *out_pos = pos;
      return;
    }
    if (tile + 128 >= nmax) {  // the step reached the edge
      *cells += nmax;
      *out_max = mx;
      *out_pos = pos;
      return;
    }
    prev_s = __shfl_sync(0xffffffffu, ts[3], 31);
    prev_m = mx;
    prev_pos = pos;
  }
}

// The position of a direction's maximum when the maximum itself is already
// known (the gate's, for a candidate whose extensions ended inside the gate):
// the earliest cell whose running sum equals it -- the cell where the running
// maximum first reached it, which lies before the dropping cell.  One sum scan
// per 32 cells and a ballot; no maximum scan.  Right: the cell's offset (-1
// when the maximum is 0); left: offset + 1 (0 when it is 0).
template <bool LEFT>
__device__ __forceinline__ int32_t exact_argmax(const uint8_t *ref, const uint8_t *qry, const int32_t *sub,
                                                uint32_t r0, uint32_t q0, uint32_t nmax, int32_t mx, uint32_t lane) {
  if (mx <= 0) return LEFT ? 0 : -1;
  int32_t prev_s = 0;
  for (uint32_t tile = 0; tile < nmax; tile += 32) {
    const uint32_t k = tile + lane;
    int32_t sc = 0;
    if (k < nmax) {
      const uint32_t rc = LEFT ? ref[r0 - 1 - k] : ref[r0 + k];
      const uint32_t qc = LEFT ? qry[q0 - 1 - k] : qry[q0 + k];
      sc = sub[rc * kNuc + qc];
    }
    const int32_t ts = (int32_t)((uint32_t)warp_incl_sum(sc, lane) + (uint32_t)prev_s);
    const uint32_t at = __ballot_sync(0xffffffffu, k < nmax && ts == mx);
    if (at) return (int32_t)(__ffs(at) - 1 + tile) + (LEFT ? 1 : 0);
    prev_s = __shfl_sync(0xffffffffu, ts, 31);
  }
  return LEFT ? 0 : -1;  // not reached for a maximum of this extension
}

constexpr int kExactThreads = 128;

__global__ void __launch_bounds__(kExactThreads) exact_kernel(ExactArgs a) {
  __shared__ int32_t sub[64];
  if (threadIdx.x < 64) sub[threadIdx.x] = a.sub[threadIdx.x];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t ncand = min(a.tot->cand, a.cand_cap);
  unsigned long long cells_acc = 0;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  for (uint32_t i = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; i < ncand; i += warps) {
    Cand cd = a.cand[i];
    const bool done = (cd.call & kDoneFlag) != 0;  // long_kernel extended it: maxima and positions known
    const bool is_long = !done && (cd.call & kLongFlag) != 0;
    CallDev call = a.calls[cd.call & ~(kLongFlag | kDoneFlag)];
    const uint8_t *qry = a.qbuf + call.qoff;
    uint32_t q0 = cd.q0 - call.qoff, r0 = cd.r0;
    unsigned long long cells = 0;
    int32_t rmax, rpos, lmax, lpos;
    if (done) {
      rmax = cd.rmax;
      lmax = cd.lmax;
      rpos = cd.rpos;
      lpos = cd.lpos;
    } else if (is_long) {  // reached the gate's cap: long runs, four cells per lane
      exact_dir4<false>(a.ref, qry, sub, a.xdrop, r0, q0, min(a.rlen - r0, call.qlen - q0), lane, &rmax, &rpos,
                        &cells);
      exact_dir4<true>(a.ref, qry, sub, a.xdrop, r0, q0, min(r0, q0), lane, &lmax, &lpos, &cells);
    } else {  // both maxima came from the gate; only their positions are left to find
      rmax = cd.rmax;
      lmax = cd.lmax;
      rpos = exact_argmax<false>(a.ref, qry, sub, r0, q0, min(a.rlen - r0, call.qlen - q0), rmax, lane);
      lpos = exact_argmax<true>(a.ref, qry, sub, r0, q0, min(r0, q0), lmax, lane);
    }
    if (is_long) cells_acc += cells;
    int32_t total = (int32_t)((uint32_t)rmax + (uint32_t)lmax);
    int32_t extent = (int32_t)((uint32_t)rpos + (uint32_t)lpos);
    int32_t T = a.hspthresh;
    int32_t T3 = (int32_t)((uint32_t)T * 3u);
    double entropy = 1.0;
    if (total >= T && total <= T3 && a.noentropy == 0) {
      uint32_t rs = r0 - (uint32_t)lpos, qs = q0 - (uint32_t)lpos;
      int32_t positions = (int32_t)((uint32_t)extent + 1u);
      unsigned long long packed = 0;  // four 16-bit match counters, packed as the reference packs them
      for (int32_t j = (int32_t)lane; j < positions; j += 32) {
        uint32_t x = a.ref[rs + (uint32_t)j], y = qry[qs + (uint32_t)j];
        if (x == y && x < 4) packed += 1ull << (16 * x);
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) packed += __shfl_xor_sync(0xffffffffu, packed, d);
      int32_t c[4] = {(int32_t)(packed & 0xFFFF), (int32_t)((packed >> 16) & 0xFFFF),
                      (int32_t)((packed >> 32) & 0xFFFF), (int32_t)((packed >> 48) & 0xFFFF)};
      if (c[0] + c[1] + c[2] + c[3] >= 20) {
        double denom = (double)((int32_t)((uint32_t)extent + 1u));
        double ent = 0.0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          double pr = __ddiv_rn((double)c[j], denom);
          double lg = c[j] != 0 ? hz_ln(pr) : 0.0;
          ent = __dadd_rn(ent, __dmul_rn(pr, lg));
        }
        entropy = __ddiv_rn(-ent, 1.3862943649291992);  // (double)logf(4.0f), src/gpu/mod.rs:2349-2352
      }
    }
    if (lane == 0 && sat_i32(__dmul_rn((double)__int2float_rn(total), entropy)) >= T) {
      SegmentPair h;
      h.ref_start = r0 - (uint32_t)lpos;
      h.query_start = q0 - (uint32_t)lpos;
      h.len = (uint32_t)extent;
      h.score = entropy > 0.0 ? sat_i32(__dmul_rn((double)total, entropy)) : 0;
      uint32_t at = atomicAdd(&a.tot->raw, 1u);
      if (at < a.raw_cap) {
        a.raw[at] = h;
        a.raw_scope[at] = cd.scope;
      }
    }
  }
  if (lane == 0 && cells_acc) atomicAdd(&a.tot->cells, cells_acc);
}

}  // namespace hz
