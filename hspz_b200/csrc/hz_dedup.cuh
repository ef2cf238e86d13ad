// dedup_and_order (src/hsp.rs:94-126) on the device, for every dedup scope
// of a wave at once.
//
// The raw HSPs of a wave carry their scope.  A stable LSD radix sort of an
// index permutation, one 32-bit field at a time from least to most
// significant, orders them by (scope, diagonal, ref_start, len, score
// descending) -- hspComp within each scope.  A record is kept when it starts
// its scope or is not contained in the previous INPUT record (hspEqual
// compares against the previous element, not the last kept one).  The kept
// records are then sorted by (scope, query_start, ref_start, len, score
// descending) -- hspCompLastz within each scope.  Both orders are total over
// the four fields, so the result equals the reference's stable sorts.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "hz_device.cuh"
#include "hz_scan.cuh"

namespace hz {

enum DedupField : int { kScoreDesc = 0, kLen = 1, kRefStart = 2, kDiag = 3, kScope = 4, kQueryStart = 5 };

// Output record of a wave: the scope and the HSP.
struct ScopedHspOut {
  uint32_t scope;
  SegmentPair h;
};

__global__ void iota_kernel(uint32_t *__restrict__ p, uint32_t n) {
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = i;
}

__device__ __forceinline__ uint32_t field_key(const SegmentPair &h, uint32_t scope, int field) {
  switch (field) {
    case kScoreDesc: return ~((uint32_t)h.score ^ 0x80000000u);  // larger score sorts first
    case kLen: return h.len;
    case kRefStart: return h.ref_start;
    case kDiag: return h.ref_start - h.query_start;  // wrapping u32 diagonal (src/hsp.rs:49-51)
    case kScope: return scope;
    default: return h.query_start;
  }
}

__global__ void gather_key_kernel(const SegmentPair *__restrict__ raw, const uint32_t *__restrict__ raw_scope,
                                  const uint32_t *__restrict__ perm, uint32_t n, int field,
                                  uint32_t *__restrict__ keys) {
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t r = perm[i];
    keys[i] = field_key(raw[r], raw_scope[r], field);
  }
}

// hspEqual (src/hsp.rs:83-87): same diagonal and one [start, start+len]
// reference interval inside the other, with wrapping ends.
__device__ __forceinline__ bool contained_dev(const SegmentPair &x, const SegmentPair &y) {
  uint32_t xe = x.ref_start + x.len, ye = y.ref_start + y.len;
  return (x.ref_start - x.query_start) == (y.ref_start - y.query_start) &&
         ((x.ref_start >= y.ref_start && xe <= ye) || (y.ref_start >= x.ref_start && ye <= xe));
}

__global__ void keep_flag_kernel(const SegmentPair *__restrict__ raw, const uint32_t *__restrict__ raw_scope,
                                 const uint32_t *__restrict__ perm, uint32_t n, uint32_t *__restrict__ keep) {
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t r = perm[i];
    bool k = true;
    if (i > 0) {
      uint32_t q = perm[i - 1];
      k = raw_scope[q] != raw_scope[r] || !contained_dev(raw[q], raw[r]);
    }
    keep[i] = k;
  }
}

__global__ void compact_perm_kernel(const uint32_t *__restrict__ perm, const uint32_t *__restrict__ keep_excl,
                                    const uint32_t *__restrict__ keep_flag, uint32_t n, uint32_t *__restrict__ out) {
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    if (keep_flag[i]) out[keep_excl[i]] = perm[i];
}

__global__ void emit_scoped_kernel(const SegmentPair *__restrict__ raw, const uint32_t *__restrict__ raw_scope,
                                   const uint32_t *__restrict__ perm, uint32_t n, ScopedHspOut *__restrict__ out) {
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t r = perm[i];
    out[i] = ScopedHspOut{raw_scope[r], raw[r]};
  }
}

}  // namespace hz
