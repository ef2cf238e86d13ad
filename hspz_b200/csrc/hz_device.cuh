// Device-side types and helpers shared by the hspz_b200 kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hz {

constexpr uint32_t kInvalidKmer = 1u << 31;  // src/seed.rs:27
constexpr uint32_t kNoBucket = 0xFFFFFFFFu;  // slot of an invalid query window
constexpr int kNuc = 8;                      // device alphabet size
constexpr int kMaxCare = 16;

// Spaced seed: `size` bases wide, `kmer_size` care positions
// (src/seed.rs:34-79).  Every care position admits a transition, as
// Shape::parse rewrites custom patterns to all-'T'.
struct ShapeDev {
  uint32_t size;
  uint32_t kmer_size;
  uint32_t pos[kMaxCare];
  // the care positions as runs of consecutive bases, in care order
  uint32_t nruns;
  uint32_t is_12of19;  // the pattern is 12of19's (TTT0T00TT00T0T0TTTT): kmer_12of19 applies
  uint32_t run_start[kMaxCare];
  uint32_t run_len[kMaxCare];
};

// Everything the extension needs besides sequence and anchors.
struct ExtendParams {
  int32_t sub[64];     // 8x8 matrix in the device alphabet (src/scoring.rs:41-120)
  int32_t xdrop;
  int32_t hspthresh;
  uint32_t noentropy;
  uint32_t rlen;       // reference block length
  uint32_t qlen;       // query block length
};

// SegmentPair (src/hsp.rs:31-41): 16 bytes, 16-byte aligned.
struct __align__(16) SegmentPair {
  uint32_t ref_start;
  uint32_t query_start;
  uint32_t len;
  int32_t score;
};

// A raw (pre-dedup) HSP tagged with its dedup scope.
struct __align__(16) ScopedHsp {
  SegmentPair h;
};

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Rust `f64 as i32`: truncation toward zero, saturating, NaN -> 0.
__device__ __forceinline__ int32_t sat_i32(double v) {
  if (v != v) return 0;
  if (v >= 2147483647.0) return 2147483647;
  if (v <= -2147483648.0) return (int32_t)0x80000000u;
  return __double2int_rz(v);
}

// hspZ's own natural log (src/gpu/kernels.rs:1879-1908): an atanh series
// over the reduced mantissa.  Every operation is an explicit
// round-to-nearest intrinsic so nothing is contracted into an FMA; the CPU
// oracle runs the identical sequence, which makes the entropy bit-exact.
__device__ __forceinline__ double hz_ln(double x) {
  const double kLn2 = 0x1.62e42fefa39efp-1;
  const double kSqrt2 = 0x1.6a09e667f3bcdp+0;
  // 1/3, 1/5, ..., 1/15 correctly rounded
  const double c3 = 0x1.5555555555555p-2, c5 = 0x1.999999999999ap-3, c7 = 0x1.2492492492492p-3,
               c9 = 0x1.c71c71c71c71cp-4, c11 = 0x1.745d1745d1746p-4, c13 = 0x1.3b13b13b13b14p-4,
               c15 = 0x1.1111111111111p-4;
  long long bits = __double_as_longlong(x);
  int ex = (int)((bits >> 52) & 0x7FF) - 1023;
  double m = __longlong_as_double((bits & 0x000FFFFFFFFFFFFFLL) | 0x3FF0000000000000LL);
  if (m > kSqrt2) {
    m = __dmul_rn(m, 0.5);
    ex += 1;
  }
  double s = __ddiv_rn(__dsub_rn(m, 1.0), __dadd_rn(m, 1.0));
  double z = __dmul_rn(s, s);
  double t = __dadd_rn(c13, __dmul_rn(z, c15));
  t = __dadd_rn(c11, __dmul_rn(z, t));
  t = __dadd_rn(c9, __dmul_rn(z, t));
  t = __dadd_rn(c7, __dmul_rn(z, t));
  t = __dadd_rn(c5, __dmul_rn(z, t));
  t = __dadd_rn(c3, __dmul_rn(z, t));
  double poly = __dadd_rn(1.0, __dmul_rn(z, t));
  return __dadd_rn(__dmul_rn(__dmul_rn(2.0, s), poly), __dmul_rn((double)ex, kLn2));
}

}  // namespace hz
