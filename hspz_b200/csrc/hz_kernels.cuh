// The seed-and-filter kernels: encoding, on-device seed table, seed lookup,
// compaction of hit-bearing seeds, the MAX_HITS chunk walk, hit expansion
// and the X-drop extension.  Semantics follow hspZ src/gpu/kernels.rs and
// src/gpu/mod.rs (cited per kernel); layouts are this library's own.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "hz_device.cuh"

namespace hz {

// ---------------------------------------------------------------------------
// Encoding.  ASCII -> device alphabet for the forward block and, in the same
// pass, for its reverse complement (encode(REV_COMP[c]) read backwards).
// src/sequence.rs:66-86, 212-230.

__constant__ uint8_t c_enc[256];
__constant__ uint8_t c_enc_rc[256];

__global__ void encode_kernel(const uint8_t *__restrict__ ascii, uint64_t n, uint8_t *__restrict__ fwd,
                              uint8_t *__restrict__ rc) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x * 4;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4; i < n; i += stride) {
    if (i + 4 <= n && ((reinterpret_cast<uintptr_t>(ascii + i) & 3) == 0)) {
      uint32_t w = *reinterpret_cast<const uint32_t *>(ascii + i);
      uint32_t f = 0;
#pragma unroll
      for (int b = 0; b < 4; b++) f |= (uint32_t)c_enc[(w >> (8 * b)) & 0xFF] << (8 * b);
      *reinterpret_cast<uint32_t *>(fwd + i) = f;
#pragma unroll
      for (int b = 0; b < 4; b++) rc[n - 1 - (i + b)] = c_enc_rc[(w >> (8 * b)) & 0xFF];
    } else {
      for (uint64_t j = i; j < i + 4 && j < n; j++) {
        uint8_t c = ascii[j];
        fwd[j] = c_enc[c];
        rc[n - 1 - j] = c_enc_rc[c];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Spaced-seed hash on device codes: INVALID unless every base of the window
// is uppercase ACGT (code < 4); else the care digits, first care position
// most significant.  src/seed.rs:88-101.

__device__ __forceinline__ uint32_t kmer_at(const uint8_t *__restrict__ codes, uint64_t pos,
                                            const ShapeDev &sh) {
  uint32_t bad = 0;
  for (uint32_t i = 0; i < sh.size; i++) bad |= codes[pos + i] & 0xFCu;
  if (bad) return kInvalidKmer;
  uint32_t kmer = 0;
  for (uint32_t t = 0; t < sh.kmer_size; t++) kmer = (kmer << 2) + codes[pos + sh.pos[t]];
  return kmer;
}

// ---------------------------------------------------------------------------
// Seed table on device (SeedTable::build, src/seed.rs:135-180): k-mers of
// the strided reference positions, compaction of the valid ones in position
// order, a stable radix sort by k-mer (so each bucket stays in ascending
// position order), and the inclusive bucket counts.

__global__ void ref_kmer_kernel(const uint8_t *__restrict__ codes, uint64_t num_steps, uint64_t start_offset,
                                uint32_t step, ShapeDev sh, uint32_t *__restrict__ kmers,
                                uint32_t *__restrict__ valid) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < num_steps; i += stride) {
    uint32_t k = kmer_at(codes, start_offset + i * step, sh);
    kmers[i] = k;
    valid[i] = k != kInvalidKmer;
  }
}

__global__ void ref_compact_kernel(const uint32_t *__restrict__ kmers, const uint32_t *__restrict__ excl,
                                   uint64_t num_steps, uint64_t start_offset, uint32_t step,
                                   uint32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                                   uint32_t *__restrict__ hist) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < num_steps; i += stride) {
    uint32_t k = kmers[i];
    if (k != kInvalidKmer) {
      uint32_t at = excl[i];
      keys[at] = k;
      vals[at] = (uint32_t)(start_offset + i * step);
      atomicAdd(&hist[k], 1u);
    }
  }
}

// inclusive = exclusive + count (index_table, src/seed.rs:162-164)
__global__ void add_counts_kernel(uint32_t *__restrict__ excl_inout, const uint32_t *__restrict__ counts,
                                  uint64_t n) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    excl_inout[i] += counts[i];
}

// ---------------------------------------------------------------------------
// Seed lookup (find_num_hits, src/gpu/kernels.rs:70-115) for the seeds of one
// call.  A call's seed list is laid out as `per_pos` slots per query
// position: slot 0 is the exact k-mer, slot 1+t its transition variant
// kmer ^ (2 << 2t) (src/seed.rs:107-123).  Invalid windows keep their slots
// with zero hits, which leaves every hit-space boundary of the MAX_HITS walk
// unchanged (their inclusive prefix repeats the preceding seed's).
//
// Per slot: cnt = bucket size, or 0 above the occurrence cap; bstart = the
// bucket's first pos_table index, kNoBucket for an invalid window.
__global__ void seed_count_kernel(const uint8_t *__restrict__ qry, uint32_t start, uint32_t span,
                                  uint32_t per_pos, ShapeDev sh, const uint32_t *__restrict__ index_table,
                                  uint32_t occ_cap, uint32_t *__restrict__ cnt, uint32_t *__restrict__ bstart,
                                  unsigned long long *__restrict__ n_valid) {
  uint32_t valid_here = 0;
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < span; p += stride) {
    uint32_t kmer = kmer_at(qry, (uint64_t)start + p, sh);
    uint64_t o = (uint64_t)p * per_pos;
    if (kmer == kInvalidKmer) {
      for (uint32_t v = 0; v < per_pos; v++) {
        cnt[o + v] = 0;
        bstart[o + v] = kNoBucket;
      }
      continue;
    }
    valid_here++;
    for (uint32_t v = 0; v < per_pos; v++) {
      uint32_t k = v == 0 ? kmer : kmer ^ (2u << (2 * (v - 1)));
      uint32_t end = __ldg(index_table + k);
      uint32_t beg = k > 0 ? __ldg(index_table + k - 1) : 0u;
      uint32_t c = end - beg;
      if (occ_cap && c > occ_cap) c = 0;
      cnt[o + v] = c;
      bstart[o + v] = beg;
    }
  }
  // one atomic per warp
  for (int d = 16; d > 0; d >>= 1) valid_here += __shfl_down_sync(0xffffffffu, valid_here, d);
  if ((threadIdx.x & 31) == 0 && valid_here) atomicAdd(n_valid, (unsigned long long)valid_here);
}

// The same lookup for host-uploaded seeds (upload_seeds, src/gpu/mod.rs:1246):
// seed = kmer << 32 | query position.
__global__ void seed_count_uploaded_kernel(const uint64_t *__restrict__ seeds, uint64_t n,
                                           const uint32_t *__restrict__ index_table, uint32_t occ_cap,
                                           uint32_t index_len, uint32_t max_pos, uint32_t *__restrict__ cnt,
                                           uint32_t *__restrict__ bstart, uint32_t *__restrict__ bad) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint64_t s = seeds[i];
    uint32_t k = (uint32_t)(s >> 32), pos = (uint32_t)s;
    if (k >= index_len || pos > max_pos) {  // would read outside the tables / query
      atomicOr(bad, 1u);
      cnt[i] = 0;
      bstart[i] = kNoBucket;
      continue;
    }
    uint32_t end = __ldg(index_table + k);
    uint32_t beg = k > 0 ? __ldg(index_table + k - 1) : 0u;
    uint32_t c = end - beg;
    if (occ_cap && c > occ_cap) c = 0;
    cnt[i] = c;
    bstart[i] = beg;
  }
}

// Pairs (hit count, non-empty flag) for the combined scan.
__global__ void pair_kernel(const uint32_t *__restrict__ cnt, uint64_t n, uint2 *__restrict__ pairs) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t c = cnt[i];
    pairs[i] = make_uint2(c, c > 0);
  }
}

// Compaction of the hit-bearing seeds, in seed order: entry e gets the
// inclusive hit prefix, the query position and the bucket start.
__global__ void seed_compact_kernel(const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ bstart,
                                    const uint2 *__restrict__ excl, uint64_t n, uint32_t per_pos,
                                    uint32_t start, const uint64_t *__restrict__ uploaded,
                                    uint32_t *__restrict__ c_incl, uint32_t *__restrict__ c_qpos,
                                    uint32_t *__restrict__ c_bstart) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t c = cnt[i];
    if (c == 0) continue;
    uint2 ex = excl[i];
    uint32_t e = ex.y;
    c_incl[e] = ex.x + c;
    c_qpos[e] = uploaded ? (uint32_t)uploaded[i] : start + (uint32_t)(i / per_pos);
    c_bstart[e] = bstart[i];
  }
}

// ---------------------------------------------------------------------------
// MAX_HITS chunk walk (chunk_limits, src/gpu/mod.rs:2394-2420) in hit space.
// With num_iter = num_hits / max_hits + 1, each cut is the largest cumulative
// hit count below the running limit; cuts are taken over the compacted
// inclusive prefixes (the zero-hit seeds in between repeat those values).
// Output: bounds[0..num_iter] with bounds[0] = 0 and bounds[num_iter] =
// num_hits; chunk c covers hits [bounds[c], bounds[c+1]).  *status = 1 when
// the very first seed alone holds >= max_hits hits, where the reference's
// walk has no valid cut (its lower_bound - 1 underflows).
__global__ void chunk_walk_kernel(const uint32_t *__restrict__ c_incl, uint32_t n_entries, uint32_t num_hits,
                                  uint32_t max_hits, uint32_t first_seed_hits, uint32_t *__restrict__ bounds,
                                  uint32_t *__restrict__ status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t num_iter = num_hits / max_hits + 1;
  bounds[0] = 0;
  *status = 0;
  if (first_seed_hits >= max_hits) {
    *status = 1;
    return;
  }
  uint32_t limit = max_hits;
  for (uint32_t it = 1; it < num_iter; it++) {
    uint32_t lo = 0, hi = n_entries;  // first entry with c_incl >= limit
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      if (c_incl[mid] < limit) lo = mid + 1; else hi = mid;
    }
    uint32_t b = lo == 0 ? 0u : c_incl[lo - 1];
    bounds[it] = b;
    limit = b + max_hits;
  }
  bounds[num_iter] = num_hits;
}

// ---------------------------------------------------------------------------
// Hit expansion (find_hits_dense, src/gpu/kernels.rs:421-465), load-balanced
// by merge path: a block owns a tile of consecutive hits, finds the
// compacted seeds that cover it, stages their prefixes in shared memory and
// gives every thread one hit at a time.  Anchors are the END of the seed
// window on both sides (pos + seed_size, kernels.rs:397-401), packed as
// ref | query << 32.  Adjacent hits of one seed read adjacent pos_table words.

constexpr int kExpandThreads = 256;
constexpr int kExpandTile = 2048;

__global__ void __launch_bounds__(kExpandThreads) expand_kernel(
    const uint32_t *__restrict__ c_incl, const uint32_t *__restrict__ c_qpos,
    const uint32_t *__restrict__ c_bstart, uint32_t n_entries, const uint32_t *__restrict__ pos_table,
    uint32_t hit_lo, uint32_t hit_hi, uint32_t seed_size, uint64_t *__restrict__ anchors) {
  __shared__ uint32_t s_incl[kExpandTile + 1];
  __shared__ uint32_t s_qpos[kExpandTile + 1];
  __shared__ uint32_t s_bst[kExpandTile + 1];
  __shared__ uint32_t s_range[2];
  uint32_t t0 = hit_lo + blockIdx.x * kExpandTile;
  if (t0 >= hit_hi) return;
  uint32_t t1 = min(t0 + (uint32_t)kExpandTile, hit_hi);
  if (threadIdx.x < 2) {
    uint32_t h = threadIdx.x == 0 ? t0 : t1 - 1;
    uint32_t lo = 0, hi = n_entries;  // first entry with c_incl > h
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      if (c_incl[mid] <= h) lo = mid + 1; else hi = mid;
    }
    s_range[threadIdx.x] = lo;
  }
  __syncthreads();
  uint32_t e0 = s_range[0], e1 = s_range[1];
  uint32_t ne = e1 - e0 + 1;  // <= tile size: every entry in between owns >= 1 hit of the tile
  for (uint32_t i = threadIdx.x; i < ne; i += blockDim.x) {
    s_incl[i] = c_incl[e0 + i];
    s_qpos[i] = c_qpos[e0 + i];
    s_bst[i] = c_bstart[e0 + i];
  }
  __syncthreads();
  for (uint32_t h = t0 + threadIdx.x; h < t1; h += blockDim.x) {
    uint32_t lo = 0, hi = ne;
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      if (s_incl[mid] <= h) lo = mid + 1; else hi = mid;
    }
    uint32_t excl = (e0 + lo) == 0 ? 0u : (lo == 0 ? c_incl[e0 - 1] : s_incl[lo - 1]);
    uint32_t j = h - excl;
    uint32_t r = __ldg(pos_table + s_bst[lo] + j) + seed_size;
    uint32_t q = s_qpos[lo] + seed_size;
    anchors[h - hit_lo] = (uint64_t)r | ((uint64_t)q << 32);
  }
}

// ---------------------------------------------------------------------------
// Ungapped X-drop extension of one hit, thread-per-hit scalar form of
// find_hsps (src/gpu/kernels.rs:1279-1406 right, :1417-1543 left).
// Right cells (r+k, q+k), left cells (r-1-k, q-1-k).  Per cell S += sub;
// M' = max(M, S) includes the cell; stop at the first cell with M' - S >
// xdrop and keep the maximum from BEFORE it; ties keep the earliest cell.
// Right position starts at -1 (offset of the best cell), left at 0 (bases
// taken).  All sums wrap like the reference's i32.

struct ExtResult {
  int32_t total;
  int32_t rpos;
  int32_t lpos;
  uint32_t cells;
};

__device__ __forceinline__ ExtResult extend_one(const uint8_t *__restrict__ ref, const uint8_t *__restrict__ qry,
                                                const int32_t *__restrict__ sub, const ExtendParams &p,
                                                uint32_t r, uint32_t q) {
  ExtResult o;
  uint32_t cells = 0;
  // right
  int32_t S = 0, M = 0, pos = -1;
  uint32_t n = min(p.rlen - r, p.qlen - q);
  uint32_t k = 0;
  for (; k < n; k++) {
    S = (int32_t)((uint32_t)S + (uint32_t)sub[ref[r + k] * kNuc + qry[q + k]]);
    int32_t Mn = max(M, S);
    if ((int32_t)((uint32_t)Mn - (uint32_t)S) > p.xdrop) {
      k++;
      break;
    }
    if (S > M) {
      M = S;
      pos = (int32_t)k;
    }
  }
  cells += k;
  int32_t rmax = M;
  o.rpos = pos;
  // left
  S = 0;
  M = 0;
  pos = 0;
  n = min(r, q);
  for (k = 0; k < n; k++) {
    S = (int32_t)((uint32_t)S + (uint32_t)sub[ref[r - 1 - k] * kNuc + qry[q - 1 - k]]);
    int32_t Mn = max(M, S);
    if ((int32_t)((uint32_t)Mn - (uint32_t)S) > p.xdrop) {
      k++;
      break;
    }
    if (S > M) {
      M = S;
      pos = (int32_t)(k + 1);
    }
  }
  cells += k;
  o.lpos = pos;
  o.total = (int32_t)((uint32_t)rmax + (uint32_t)M);
  o.cells = cells;
  return o;
}

// Entropy correction and final acceptance (src/gpu/kernels.rs:1555-1701).
// Returns true and fills *out when the HSP is kept.
__device__ __forceinline__ bool accept_hsp(const uint8_t *__restrict__ ref, const uint8_t *__restrict__ qry,
                                           const ExtendParams &p, uint32_t r, uint32_t q, const ExtResult &e,
                                           SegmentPair *out) {
  int32_t extent = (int32_t)((uint32_t)e.rpos + (uint32_t)e.lpos);
  int32_t T = p.hspthresh;
  int32_t T3 = (int32_t)((uint32_t)T * 3u);
  double entropy = 1.0;
  if (e.total >= T && e.total <= T3 && p.noentropy == 0) {
    uint32_t rs = r - (uint32_t)e.lpos, qs = q - (uint32_t)e.lpos;
    int32_t positions = (int32_t)((uint32_t)extent + 1u);
    unsigned long long packed = 0;  // four 16-bit match counters, as the reference packs them
    for (int32_t i = 0; i < positions; i++) {
      uint32_t a = ref[rs + (uint32_t)i], b = qry[qs + (uint32_t)i];
      if (a == b && a < 4) packed += 1ull << (16 * a);
    }
    int32_t c[4] = {(int32_t)(packed & 0xFFFF), (int32_t)((packed >> 16) & 0xFFFF),
                    (int32_t)((packed >> 32) & 0xFFFF), (int32_t)((packed >> 48) & 0xFFFF)};
    if (c[0] + c[1] + c[2] + c[3] >= 20) {
      double denom = (double)((int32_t)((uint32_t)extent + 1u));
      double ent = 0.0;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        double pr = __ddiv_rn((double)c[i], denom);
        double lg = c[i] != 0 ? hz_ln(pr) : 0.0;
        ent = __dadd_rn(ent, __dmul_rn(pr, lg));
      }
      entropy = __ddiv_rn(-ent, 1.3862943649291992);  // (double)logf(4.0f), src/gpu/mod.rs:2349-2352
    }
  }
  double upper = (double)__int2float_rn(e.total);
  if (sat_i32(__dmul_rn(upper, entropy)) < T) return false;
  out->ref_start = r - (uint32_t)e.lpos;
  out->query_start = q - (uint32_t)e.lpos;
  out->len = (uint32_t)extent;
  out->score = entropy > 0.0 ? sat_i32(__dmul_rn((double)e.total, entropy)) : 0;
  return true;
}

// One thread per anchor; accepted HSPs are appended to `raw` through an
// atomic cursor (their order is irrelevant: each dedup scope is sorted on
// all four fields).  `cells` accumulates the scalar cells scored.
constexpr int kExtendThreads = 256;

__global__ void __launch_bounds__(kExtendThreads) extend_kernel(const uint8_t *__restrict__ ref,
                                                                const uint8_t *__restrict__ qry,
                                                                const uint64_t *__restrict__ anchors,
                                                                uint32_t n_hits, ExtendParams p,
                                                                SegmentPair *__restrict__ raw, uint32_t raw_cap,
                                                                uint32_t *__restrict__ raw_count,
                                                                unsigned long long *__restrict__ cells_out) {
  __shared__ int32_t sub[64];
  if (threadIdx.x < 64) sub[threadIdx.x] = p.sub[threadIdx.x];
  __syncthreads();
  unsigned long long cells = 0;
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_hits; i += stride) {
    uint64_t a = anchors[i];
    uint32_t r = (uint32_t)a, q = (uint32_t)(a >> 32);
    if (r > p.rlen || q > p.qlen) continue;  // unreachable for validated tables and seeds
    ExtResult e = extend_one(ref, qry, sub, p, r, q);
    cells += e.cells;
    SegmentPair h;
    if (accept_hsp(ref, qry, p, r, q, e, &h)) {
      uint32_t at = atomicAdd(raw_count, 1u);
      if (at < raw_cap) raw[at] = h;
    }
  }
  for (int d = 16; d > 0; d >>= 1) cells += __shfl_down_sync(0xffffffffu, cells, d);
  if ((threadIdx.x & 31) == 0 && cells) atomicAdd(cells_out, cells);
}

}  // namespace hz
