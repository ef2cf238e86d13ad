// Gate kernel of the wave pipeline (included by hz_wave.cuh).
//
// A persistent grid of independent warps: each warp takes tiles of TW
// consecutive wave hits from a device work queue and, with warp-level
// synchronisation only (no block barrier, so one warp's memory latency in
// its tile setup overlaps the other warps' scoring),
//   (1) recomputes the seeds of the positions covering the tile and records
//       the (position, seed) slots that overlap it, issuing the bucket
//       lookups of several seeds at once;
//   (2) gives every hit its slot by a warp max-scan of slot-start marks and
//       stores, per hit, the reference and query anchors, the distances to
//       the sequence edges and the call -- so that a lane picking up a hit
//       later touches shared memory only;
//   (3) runs the X-drop score gate thread-per-hit, first all right
//       extensions of the tile and then all left extensions.  Before each
//       pass the warp gathers every hit's first eight cells of both
//       sequences, so a lane's first step scores from shared memory while
//       the words of its second step load; each lane refills from the tile
//       when its extension ends, so extensions of different lengths do not
//       idle the warp, and it fetches the words of its next eight cells one
//       step ahead.
// The kernel leans on L1: a hit's reference and query lines, brought in when
// its first cells are gathered, serve the loads of its later steps.  So the
// per-warp shared memory is kept small enough for four blocks per SM to
// leave ~90 KB of L1 (with 28 KB the gate runs ~1.5x slower).
// Anchors are the END of the seed window on both sides (pos + seed_size,
// src/gpu/kernels.rs:397-401).  A hit becomes a candidate when
// (i32)(f32)(right max + left max) >= hspthresh -- the reference gate's bound
// (src/gpu/kernels.rs:1048-1052), never below the final score since the
// entropy factor is <= 1 -- or when an extension runs past `cap` cells
// ("long"; the exact kernel redoes it warp-wide).
#pragma once

namespace hz {

constexpr int kGateThreads = 256;
constexpr int kGateWarps = kGateThreads / 32;

// Shared memory of one warp's tile.  The per-tile setup arrays and the
// per-pass "first eight cells" arrays are never live at the same time.
template <int TW>
struct WarpTile {
  union {
    struct {
      uint32_t slot_bst[TW];  // pos_table index of the slot's first in-tile hit
      uint32_t slot_q[TW];    // query anchor (absolute)
      uint32_t slot_call[TW];
      uint32_t hit_slot[TW];  // first hit of the hit's slot + 1 (mark, then max-scan)
    } setup;
    struct {
      uint4 first[TW];  // first eight cells: reference words a, b; query words a, b
    } pass;
  } u;
  uint32_t hit_r[TW];     // reference anchor
  uint32_t hit_q[TW];     // query anchor (absolute)
  uint32_t hit_n[TW];     // cells to the right edge | cells to the left edge << 16 (each saturated)
  uint32_t hit_call[TW];
  int32_t hit_rmax[TW];   // right-extension maximum, or kSpilled
  uint16_t hit_rcells[TW];
};

template <int TW>
struct GateSmem {
  int32_t sub[64];
  WarpTile<TW> warp[kGateWarps];
};
constexpr int32_t kSpilled = -1;  // a right maximum is never negative

struct GateArgs {
  WaveIn w;
  const unsigned long long *np_excl;
  const uint32_t *np_pos;
  const uint32_t *np_kmer;  // k-mer of each position with hits (np_emit_kernel), or null
  const unsigned long long *scope_lo;
  uint32_t scope_cap;  // entries of scope_lo (a wave with more scopes is rerun)
  WaveTotals *tot;
  int32_t sub[64];
  int32_t xdrop;
  int32_t hspthresh;
  uint32_t cap;  // cells per direction before a hit goes to the exact kernel (multiple of 8, < 65536)
  Cand *cand;
  uint32_t cand_cap;
  const uint32_t *tile_first;  // first position with hits of each tile (tile_table_kernel)
  const uint32_t *tile_call;   // call of that position
  // 7 * (largest substitution score) <= xdrop: no cell within seven cells
  // after a dropping cell can raise the maximum, so an extension that drops
  // inside an eight-cell group ends with the group's final maximum
  uint32_t late_max_safe;
  // 2 * cap * (largest substitution score) < 2^24: every gate total is exact
  // in f32, so (i32)(f32)total >= hspthresh is total >= hspthresh
  uint32_t total_exact;
};

__device__ __forceinline__ const uint32_t *word_ptr(const uint8_t *p) {
  return reinterpret_cast<const uint32_t *>(reinterpret_cast<uintptr_t>(p) & ~(uintptr_t)3);
}

// Inclusive max-scan of the slot marks over the warp's tile.
template <int TW>
__device__ __forceinline__ void mark_scan(WarpTile<TW> &wt, uint32_t nt, uint32_t lane) {
  constexpr int PER = TW / 32;
  uint32_t *mark = wt.u.setup.hit_slot;
  const uint32_t base = lane * PER;
  uint32_t run = 0;
#pragma unroll
  for (int i = 0; i < PER; i++)
    if (base + i < nt) run = max(run, mark[base + i]);
  uint32_t incl = run;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t up = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= (uint32_t)d) incl = max(incl, up);
  }
  uint32_t carry = __shfl_up_sync(0xffffffffu, incl, 1);
  if (lane == 0) carry = 0;
#pragma unroll
  for (int i = 0; i < PER; i++)
    if (base + i < nt) {
      carry = max(carry, mark[base + i]);
      mark[base + i] = carry;
    }
}

__device__ __forceinline__ uint32_t scope_of(const unsigned long long *scope_lo, uint32_t nscopes,
                                             unsigned long long h) {
  uint32_t lo = 0, hi = nscopes;  // last scope with scope_lo <= h
  while (hi - lo > 1) {
    uint32_t m = (lo + hi) >> 1;
    if (scope_lo[m] <= h) lo = m; else hi = m;
  }
  return lo;
}

// The eight bytes [p, p+8) (right) or [p-8, p) reversed (left) as two words,
// cell 0 in the low byte, plus the word the next step continues from.
template <bool LEFT>
__device__ __forceinline__ void first_group(const uint8_t *seq, uint32_t p, uint32_t *a, uint32_t *b,
                                            uint32_t *carry) {
  const uint32_t sh = (p & 3u) * 8u;
  if (!LEFT) {
    const uint32_t *w = word_ptr(seq + p);
    uint32_t w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2);
    *a = __funnelshift_r(w0, w1, sh);
    *b = __funnelshift_r(w1, w2, sh);
    *carry = w2;
  } else {
    const uint32_t *w = word_ptr(seq + p - 8);
    uint32_t w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2);
    *a = __byte_perm(__funnelshift_r(w1, w2, sh), 0, 0x0123);
    *b = __byte_perm(__funnelshift_r(w0, w1, sh), 0, 0x0123);
    *carry = w0;
  }
}

// Scores one cell whose byte offset into the substitution table is byte SH
// of T (extracted, zero-extended, by one byte permute); keeps every running
// sum S for the termination path and the group's smallest sum.  Since every
// running maximum M_i <= M_7, no cell of the group can have dropped when
// M_7 - min S <= xdrop.
#define HZ_CELL(T, SH, I)                                                            \
  {                                                                                  \
    int32_t sc = *reinterpret_cast<const int32_t *>(subb + __byte_perm((T), 0u, 0x4440u + (SH) / 8)); \
    S = (int32_t)((uint32_t)S + (uint32_t)sc);                                       \
    M = max(M, S);                                                                   \
    Si[I] = S;                                                                       \
    Smin = min(Smin, S);                                                             \
  }

template <int TW, bool LEFT>
__device__ __forceinline__ void gate_phase(const GateArgs &a, const char *subb, WarpTile<TW> &wt, uint32_t hi,
                                           unsigned long long h0, unsigned long long &cells_acc) {
  const uint8_t *ref = a.w.ref;
  const uint8_t *qbuf = a.w.qbuf;
  const int32_t X = a.xdrop;
  const uint32_t lane = threadIdx.x & 31;
  bool have = false, exhausted = false, capped = false;
  uint32_t t = 0, n = 0;
  int32_t S = 0, M = 0;
  uint32_t cells = 0;
  // word stream state: the group about to be scored (ra, rb, qa, qb), the
  // word the following group starts in and the two prefetched words after it
  uint32_t ra = 0, rb = 0, qa = 0, qb = 0;
  uint32_t rc = 0, r1 = 0, r2 = 0, qc = 0, q1 = 0, q2 = 0;
  const uint32_t *wr = nullptr, *wq = nullptr;
  uint32_t sr = 0, sq = 0;
  uint32_t cursor = 0;  // next unclaimed hit of the tile (the same in every lane)
  while (true) {
    if (!exhausted) {
      unsigned need = __ballot_sync(0xffffffffu, !have);
      if (need) {
        const uint32_t base = cursor;
        cursor += (uint32_t)__popc(need);
        if (cursor >= hi) exhausted = true;
        if (!have) {
          uint32_t mine = base + __popc(need & lanemask_lt());
          if (mine < hi && !(LEFT && wt.hit_rmax[mine] == kSpilled)) {
            have = true;
            t = mine;
            const uint32_t r0 = wt.hit_r[t], q0 = wt.hit_q[t];
            n = LEFT ? (wt.hit_n[t] >> 16) : (wt.hit_n[t] & 0xFFFFu);
            capped = n > a.cap;
            if (capped) n = a.cap;
            S = 0;
            M = 0;
            cells = 0;
            uint4 f = wt.u.pass.first[t];
            ra = f.x;
            rb = f.y;
            qa = f.z;
            qb = f.w;
            sr = r0 << 3;  // the funnel shifts use the low five bits: (r0 & 3) * 8
            sq = q0 << 3;
            // the carried word is reloaded here rather than staged: its line
            // is in L1 from the gather, and the smaller staging leaves L1 larger
            if (!LEFT) {
              wr = word_ptr(ref + r0) + 2;  // the carried word
              wq = word_ptr(qbuf + q0) + 2;
              rc = __ldg(wr);
              qc = __ldg(wq);
              r1 = __ldg(wr + 1);
              r2 = __ldg(wr + 2);
              q1 = __ldg(wq + 1);
              q2 = __ldg(wq + 2);
            } else {
              wr = word_ptr(ref + r0 - 8);  // the carried word
              wq = word_ptr(qbuf + q0 - 8);
              rc = __ldg(wr);
              qc = __ldg(wq);
              r1 = __ldg(wr - 1);
              r2 = __ldg(wr - 2);
              q1 = __ldg(wq - 1);
              q2 = __ldg(wq - 2);
            }
          }
        }
      }
    }
    // (in the left pass a refill may hand out only hits that were spilled in
    // the right pass, so an idle warp ends only once the tile is exhausted)
    if (!__any_sync(0xffffffffu, have) && exhausted) break;
    if (!have) continue;
    // ---- eight cells ----
    // codes are 0..7, so (r << 5) | (q << 2) is the byte offset of sub[r*8+q]
    const uint32_t ta = (ra << 5) | (qa << 2), tb = (rb << 5) | (qb << 2);
    // the next group from the carried and prefetched words; prefetch again
    uint32_t nra, nrb, nqa, nqb;
    if (!LEFT) {
      nra = __funnelshift_r(rc, r1, sr);
      nrb = __funnelshift_r(r1, r2, sr);
      nqa = __funnelshift_r(qc, q1, sq);
      nqb = __funnelshift_r(q1, q2, sq);
      rc = r2;
      qc = q2;
      wr += 2;
      wq += 2;
    } else {
      nra = __byte_perm(__funnelshift_r(r1, rc, sr), 0, 0x0123);
      nrb = __byte_perm(__funnelshift_r(r2, r1, sr), 0, 0x0123);
      nqa = __byte_perm(__funnelshift_r(q1, qc, sq), 0, 0x0123);
      nqb = __byte_perm(__funnelshift_r(q2, q1, sq), 0, 0x0123);
      rc = r2;
      qc = q2;
      wr -= 2;
      wq -= 2;
    }
    const int32_t Ms = M;
    int32_t Si[8];
    int32_t Smin = S;
    HZ_CELL(ta, 0, 0)
    HZ_CELL(ta, 8, 1)
    HZ_CELL(ta, 16, 2)
    HZ_CELL(ta, 24, 3)
    HZ_CELL(tb, 0, 4)
    HZ_CELL(tb, 8, 5)
    HZ_CELL(tb, 16, 6)
    HZ_CELL(tb, 24, 7)
    // first valid cell with M - S > xdrop, if the bound says there may be one
    const uint32_t v = min(n, 8u);
    uint32_t dm = 0;
    if ((int32_t)((uint32_t)M - (uint32_t)Smin) > X || n <= 8) {
      int32_t m = Ms;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        m = max(m, Si[i]);
        dm |= (uint32_t)((int32_t)((uint32_t)m - (uint32_t)Si[i]) > X) << i;
      }
      dm &= (1u << v) - 1u;
    }
    if (!dm && n > 8) {  // no drop and more cells left: advance the stream
      n -= 8;
      cells += 8;
      ra = nra;
      rb = nrb;
      qa = nqa;
      qb = nqb;
      if (n > 8) {  // words of the group after next (never beyond the padding)
        if (!LEFT) {
          r1 = __ldg(wr + 1);
          r2 = __ldg(wr + 2);
          q1 = __ldg(wq + 1);
          q2 = __ldg(wq + 2);
        } else {
          r1 = __ldg(wr - 1);
          r2 = __ldg(wr - 2);
          q1 = __ldg(wq - 1);
          q2 = __ldg(wq - 2);
        }
      }
      continue;
    }
    // The extension ends in this group: at the first valid cell with
    // M - S > xdrop (keeping the maximum from before it), or after the v
    // valid cells left before the edge or the cap.
    const uint32_t stop = dm ? (uint32_t)(__ffs(dm) - 1) : v;
    int32_t res = M;  // a drop, and no later cell of the group raised the maximum
    if (!dm || !a.late_max_safe) {  // the maximum over the cells before `stop`
      res = Ms;
#pragma unroll
      for (int i = 0; i < 8; i++)
        if ((uint32_t)i < stop) res = max(res, Si[i]);
    }
    cells += dm ? stop + 1 : v;
    const bool spill = !dm && capped;
    if (spill) {
      uint32_t at = atomicAdd(&a.tot->cand, 1u);
      if (at < a.cand_cap)
        a.cand[at] = Cand{scope_of(a.scope_lo, min(a.tot->n_scopes, a.scope_cap), h0 + t), wt.hit_r[t],
                          wt.hit_q[t], wt.hit_call[t] | kLongFlag, 0, 0};
      if (!LEFT) wt.hit_rmax[t] = kSpilled;  // the left pass skips it
    } else if (!LEFT) {
      wt.hit_rmax[t] = res;
      wt.hit_rcells[t] = (uint16_t)cells;
    } else {
      cells_acc += cells + wt.hit_rcells[t];
      int32_t total = (int32_t)((uint32_t)wt.hit_rmax[t] + (uint32_t)res);
      if (a.total_exact ? total >= a.hspthresh : sat_i32((double)__int2float_rn(total)) >= a.hspthresh) {
        uint32_t at = atomicAdd(&a.tot->cand, 1u);
        if (at < a.cand_cap)
          a.cand[at] = Cand{scope_of(a.scope_lo, min(a.tot->n_scopes, a.scope_cap), h0 + t), wt.hit_r[t],
                            wt.hit_q[t], wt.hit_call[t], wt.hit_rmax[t], res};
      }
    }
    have = false;
  }
}

// Fills the first eight cells of every hit of the warp's tile for one pass.
template <int TW, bool LEFT>
__device__ __forceinline__ void prepare_pass(const GateArgs &a, WarpTile<TW> &wt, uint32_t nt, uint32_t lane) {
  for (uint32_t i = lane; i < nt; i += 32) {
    if (LEFT && wt.hit_rmax[i] == kSpilled) continue;
    uint32_t ra, rb, rc, qa, qb, qc;
    first_group<LEFT>(a.w.ref, wt.hit_r[i], &ra, &rb, &rc);
    first_group<LEFT>(a.w.qbuf, wt.hit_q[i], &qa, &qb, &qc);
    wt.u.pass.first[i] = make_uint4(ra, rb, qa, qb);
  }
}

// Bucket lookups issued per group of seeds, so their loads are in flight
// together.
constexpr uint32_t kLookupBatch = 8;

template <int TW>
__global__ void __launch_bounds__(kGateThreads) gate_kernel(GateArgs a) {
  static_assert(TW % 32 == 0, "a warp tile is a multiple of 32 hits");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GateSmem<TW> &sm = *reinterpret_cast<GateSmem<TW> *>(smem_raw);
  if (a.tot->status & 4u) return;  // no tile table: the host reruns the wave with a larger one
  if (threadIdx.x < 64) sm.sub[threadIdx.x] = a.sub[threadIdx.x];
  __syncthreads();  // the block's only barrier
  const char *subb = reinterpret_cast<const char *>(sm.sub);
  WarpTile<TW> &wt = sm.warp[threadIdx.x >> 5];
  const uint32_t lane = threadIdx.x & 31;
  unsigned long long cells_acc = 0;
  const unsigned long long total = a.tot->hits;
  const uint32_t nz = a.tot->nz;
  const WaveIn &w = a.w;
  while (true) {
    unsigned long long j = 0;
    if (lane == 0) j = atomicAdd(&a.tot->tiles, 1ull);
    j = __shfl_sync(0xffffffffu, j, 0);
    const unsigned long long h0 = j * (unsigned long long)TW;
    if (h0 >= total) break;
    const uint32_t nt = (uint32_t)min((unsigned long long)TW, total - h0);
    // positions covering [h0, h0 + nt): the tile table gives the first; the
    // last is the one before the next tile's first, unless that one already
    // started inside this tile
    const uint32_t k0 = a.tile_first[j], k1 = a.tile_first[j + 1];
    const uint32_t e1 = (k1 >= nz || a.np_excl[k1] == h0 + nt) ? k1 - 1 : k1;
    uint32_t c = a.tile_call[j];  // calls only advance with the position
    __syncwarp();                 // the previous tile's left pass is done with the union
    for (uint32_t i = lane; i < nt; i += 32) wt.u.setup.hit_slot[i] = 0;
    __syncwarp();
    // (1) slots overlapping the tile
    for (uint32_t k = k0 + lane; k <= e1; k += 32) {
      uint32_t p = a.np_pos[k];
      while (c + 1 < w.ncalls && w.calls[c + 1].pos_off <= p) c++;
      CallDev cd = w.calls[c];
      uint32_t qpos, kmer;
      position_seed(w, cd, p, &qpos, &kmer);
      unsigned long long lo = a.np_excl[k];
      const uint32_t q_anchor = cd.qoff + qpos + w.shape.size;
      for (uint32_t v0 = 0; v0 < w.per_pos; v0 += kLookupBatch) {
        uint32_t beg[kLookupBatch], cnt[kLookupBatch];
#pragma unroll
        for (uint32_t u = 0; u < kLookupBatch; u++) {
          cnt[u] = 0;
          beg[u] = 0;
          if (v0 + u < w.per_pos) cnt[u] = bucket(w, seed_variant(kmer, v0 + u), &beg[u]);
        }
#pragma unroll
        for (uint32_t u = 0; u < kLookupBatch; u++) {
          unsigned long long hi = lo + cnt[u];
          if (cnt[u] && hi > h0 && lo < h0 + nt) {
            unsigned long long first = lo > h0 ? lo : h0;
            uint32_t s = (uint32_t)(first - h0);
            wt.u.setup.slot_bst[s] = beg[u] + (uint32_t)(first - lo);
            wt.u.setup.slot_q[s] = q_anchor;
            wt.u.setup.slot_call[s] = c;
            wt.u.setup.hit_slot[s] = s + 1;
          }
          lo = hi;
        }
      }
    }
    __syncwarp();
    // (2) per hit: slot, anchors, edge distances, call
    mark_scan<TW>(wt, nt, lane);
    __syncwarp();
    for (uint32_t i = lane; i < nt; i += 32) {
      uint32_t s = wt.u.setup.hit_slot[i] - 1;
      uint32_t r0 = __ldg(w.pos_table + wt.u.setup.slot_bst[s] + (i - s)) + w.shape.size;
      uint32_t q0 = wt.u.setup.slot_q[s];
      uint32_t hc = wt.u.setup.slot_call[s];
      const CallDev &cd = w.calls[hc];
      uint32_t nr = min(w.rlen - r0, cd.qoff + cd.qlen - q0);
      uint32_t nl = min(r0, q0 - cd.qoff);
      wt.hit_r[i] = r0;
      wt.hit_q[i] = q0;
      wt.hit_n[i] = min(nr, 0xFFFFu) | (min(nl, 0xFFFFu) << 16);
      wt.hit_call[i] = hc;
    }
    __syncwarp();
    // (3) the score gate: right pass, then left pass
    prepare_pass<TW, false>(a, wt, nt, lane);
    __syncwarp();
    gate_phase<TW, false>(a, subb, wt, nt, h0, cells_acc);
    __syncwarp();
    prepare_pass<TW, true>(a, wt, nt, lane);
    __syncwarp();
    gate_phase<TW, true>(a, subb, wt, nt, h0, cells_acc);
  }
  for (int d = 16; d > 0; d >>= 1) cells_acc += __shfl_down_sync(0xffffffffu, cells_acc, d);
  if (lane == 0 && cells_acc) atomicAdd(&a.tot->cells, cells_acc);
}

}  // namespace hz
