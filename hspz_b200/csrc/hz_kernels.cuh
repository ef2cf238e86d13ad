// Encoding and the on-device seed table.  The seed-and-filter wave itself
// lives in hz_wave.cuh.
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
    // word path only when both the load and the store are 4-byte aligned
    if (i + 4 <= n && (((reinterpret_cast<uintptr_t>(ascii + i) | reinterpret_cast<uintptr_t>(fwd + i)) & 3) == 0)) {
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
// 2-bit packing for the score gate and the seed windows.  A packed sequence is
// one logical run of 2 * half bases: the block forward in [0, half) and read
// backwards in [half, 2 * half) (base half + i is base n - 1 - i), so a left
// extension walks the reversed half forwards with the same code as a right
// one.  Every 32 bases are one 16-byte record: x, y = the ACGT codes (2 bits
// per base, base i at bits 2 (i % 16) of x for i < 16, of y above), z = the
// special mask (bit i set when base i is not uppercase ACGT -- soft-masked,
// N, other or separator -- whose code packs as 0), w = 0.  Positions past the
// block in each half are 0 and not special; extensions never score them.  One
// record per thread.
__global__ void pack2_kernel(const uint8_t *__restrict__ codes, uint64_t n, uint64_t half,
                             uint4 *__restrict__ blk) {
  const uint64_t blocks = (2 * half) / 32;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < blocks; b += stride) {
    uint32_t lo = 0, hi = 0, sp = 0;
    const uint64_t o0 = b * 32;
    const bool rev = o0 >= half;
#pragma unroll 4
    for (uint32_t i = 0; i < 32; i++) {
      const uint64_t o = (rev ? o0 - half : o0) + i;
      if (o >= n) break;
      const uint32_t c = codes[rev ? n - 1 - o : o];
      const uint32_t bits = c < 4 ? c : 0u;
      if (i < 16) lo |= bits << (2 * i);
      else hi |= bits << (2 * (i - 16));
      sp |= (uint32_t)(c >= 4) << i;
    }
    blk[b] = make_uint4(lo, hi, sp, 0u);
  }
}

// The 32 bases of a packed half that start at base p: their codes (lo: the
// first 16, hi: the next 16) and their special bits, from the two 16-byte
// records that hold them.
__device__ __forceinline__ void window32(const uint4 *__restrict__ blk, uint32_t p, uint32_t *lo, uint32_t *hi,
                                         uint32_t *sp) {
  const uint4 A = __ldg(blk + (p >> 5)), B = __ldg(blk + (p >> 5) + 1);
  const uint32_t o = p & 31u, sh = (o & 15u) << 1;
  const bool upper = o >= 16;  // the window starts in the record's second code word
  const uint32_t w0 = upper ? A.y : A.x, w1 = upper ? B.x : A.y, w2 = upper ? B.y : B.x;
  *lo = __funnelshift_r(w0, w1, sh);
  *hi = __funnelshift_r(w1, w2, sh);
  *sp = __funnelshift_r(A.z, B.z, o);
}

// ---------------------------------------------------------------------------
// Spaced-seed hash on device codes: INVALID unless every base of the window
// is uppercase ACGT (code < 4); else the care digits, first care position
// most significant.  src/seed.rs:88-101.

// The window is checked a 4-byte word at a time; the aligned words may
// reach up to three bytes before and after it, which every code buffer's
// padding covers.
__device__ __forceinline__ uint32_t kmer_at(const uint8_t *__restrict__ codes, uint64_t pos,
                                            const ShapeDev &sh) {
  const uint8_t *p = codes + pos;
  const uint32_t off = (uint32_t)(reinterpret_cast<uintptr_t>(p) & 3u);
  const uint32_t *wp = reinterpret_cast<const uint32_t *>(p - off);
  const uint32_t nbytes = off + sh.size;  // bytes from the first aligned word to the window's end
  uint32_t bad = 0;
  for (uint32_t b = 0; b < nbytes; b += 4) {
    uint32_t x = __ldg(wp + (b >> 2)) & 0xFCFCFCFCu;
    if (b == 0) x &= 0xFFFFFFFFu << (8u * off);                       // bytes before the window
    if (b + 4 > nbytes) x &= 0xFFFFFFFFu >> (8u * (b + 4 - nbytes));  // bytes after it
    bad |= x;
  }
  if (bad) return kInvalidKmer;
  uint32_t kmer = 0;
  for (uint32_t t = 0; t < sh.kmer_size; t++) kmer = (kmer << 2) + codes[pos + sh.pos[t]];
  return kmer;
}

// The same k-mer from a packed sequence (pack2_kernel's forward half), for
// patterns of at most 32 bases: the window's special bits decide validity
// with one masked test, and the care digits come out of one 64-bit window
// of codes instead of one byte load each.
__device__ __forceinline__ uint32_t kmer_packed(const uint4 *__restrict__ blk, uint32_t x, const ShapeDev &sh) {
  uint32_t lo, hi, sp;
  window32(blk, x, &lo, &hi, &sp);
  if (sp & (sh.size >= 32 ? 0xFFFFFFFFu : ((1u << sh.size) - 1u))) return kInvalidKmer;
  uint32_t kmer = 0;
  for (uint32_t t = 0; t < sh.kmer_size; t++) {
    const uint32_t p = sh.pos[t];
    const uint32_t d = p < 16 ? lo >> (2 * p) : hi >> (2 * p - 32);
    kmer = (kmer << 2) | (d & 3u);
  }
  return kmer;
}

// The k-mer of the window that starts j bases into 32 packed bases w64 (base
// i at bits 2i..2i+1), for patterns of at most 32 - j bases: the care digits
// come out a run of consecutive care positions at a time, first care
// position in the lowest bits, and one digit reversal puts it on top.
__device__ __forceinline__ uint32_t kmer_runs(uint64_t w64, uint32_t j, const ShapeDev &sh) {
  const uint64_t x = w64 >> (2 * j);
  uint32_t le = 0, at = 0;
  for (uint32_t r = 0; r < sh.nruns; r++) {
    const uint32_t len2 = 2 * sh.run_len[r];
    le |= ((uint32_t)(x >> (2 * sh.run_start[r])) & ((1u << len2) - 1u)) << at;
    at += len2;
  }
  uint32_t rv = __brev(le);
  rv = ((rv >> 1) & 0x55555555u) | ((rv & 0x55555555u) << 1);
  return rv >> (32 - 2 * sh.kmer_size);
}

// kmer_runs for the 12of19 pattern (TTT0T00TT00T0T0TTTT: runs of 3, 1, 2,
// 1, 1 and 4 care positions at bases 0, 4, 7, 11, 13 and 15) with constant
// shifts: each run's field moves to its place in one shift and one mask.
// lo, hi: 32 packed bases; j <= 13.
__device__ __forceinline__ uint32_t kmer_12of19(uint32_t lo, uint32_t hi, uint32_t j) {
  const uint32_t xlo = __funnelshift_r(lo, hi, 2 * j), xhi = hi >> (2 * j);
  const uint32_t y = __funnelshift_r(xlo, xhi, 14);  // bases 7.. of the window
  const uint32_t le = (xlo & 0x3Fu) | ((xlo >> 2) & (0x3u << 6)) | ((xlo >> 6) & (0xFu << 8)) |
                      ((xlo >> 10) & (0x3u << 12)) | ((xlo >> 12) & (0x3u << 14)) | (y & (0xFFu << 16));
  uint32_t rv = __brev(le);
  rv = ((rv >> 1) & 0x55555555u) | ((rv & 0x55555555u) << 1);
  return rv >> 8;
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

}  // namespace hz
