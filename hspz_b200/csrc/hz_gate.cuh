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
//       the sequence edges and the call, plus the first eight cells of both
//       extensions -- so that a lane picking up a hit touches shared memory
//       only;
//   (3) runs the X-drop score gate thread-per-hit: a lane scores a hit's
//       right extension and then its left extension, and takes the next hit
//       of the tile when both end, so extensions of different lengths do
//       not idle the warp.  A left extension is scored as a right extension
//       over the reversed reference and query copies, so both directions
//       run the same code: eight cells per step from two 4-byte words per
//       sequence, the words of the next step fetched one step ahead.
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
// first cells of the extensions are never live at the same time.
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
      uint4 right[TW];  // first eight cells to the right: reference words a, b; query words a, b
      uint4 left[TW];   // the same to the left, from the reversed copies
    } pass;
  } u;
  uint32_t hit_r[TW];   // reference anchor
  uint32_t hit_q[TW];   // query anchor (absolute)
  uint32_t hit_ql[TW];  // query anchor in the reversed copy of the strand
  uint32_t hit_n[TW];   // cells to the right edge | cells to the left edge << 16 (each saturated)
  uint32_t hit_call[TW];
};

template <int TW>
struct GateSmem {
  int32_t sub[64];
  WarpTile<TW> warp[kGateWarps];
};

struct GateArgs {
  WaveIn w;
  const unsigned long long *np_excl;
  const uint32_t *np_pos;
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

// The eight bytes [p, p+8) as two words, cell 0 in the low byte.
__device__ __forceinline__ void first_group(const uint8_t *seq, uint32_t p, uint32_t *a, uint32_t *b) {
  const uint32_t sh = (p & 3u) * 8u;
  const uint32_t *w = word_ptr(seq + p);
  uint32_t w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2);
  *a = __funnelshift_r(w0, w1, sh);
  *b = __funnelshift_r(w1, w2, sh);
}

// Scores the two cells whose byte offsets into the substitution table are
// bytes SH0 and SH1 of T: the running sums after each go to Si[I], Si[I+1];
// the group's running maximum M and smallest sum Smin take both at once.
// Since every cell's maximum is <= the group's final M, no cell of the group
// can have dropped when M - Smin <= xdrop.
#define HZ_PAIR(T, SH0, SH1, I)                                                            \
  {                                                                                        \
    const int32_t s0 = *reinterpret_cast<const int32_t *>(subb + (((T) >> (SH0)) & 0xFFu)); \
    const int32_t s1 = *reinterpret_cast<const int32_t *>(subb + (((T) >> (SH1)) & 0xFFu)); \
    Si[I] = (int32_t)((uint32_t)S + (uint32_t)s0);                                         \
    S = (int32_t)((uint32_t)Si[I] + (uint32_t)s1);                                         \
    Si[I + 1] = S;                                                                         \
    M = __vimax3_s32(M, Si[I], S);                                                         \
    Smin = __vimin3_s32(Smin, Si[I], S);                                                   \
  }

// Stream state of one lane's extension: the group about to be scored (ra,
// rb, qa, qb), the carried word and the two prefetched words of each
// sequence, and where the next words come from.
struct Stream {
  uint32_t ra, rb, qa, qb;
  uint32_t rc, r1, r2, qc, q1, q2;
  const uint32_t *wr, *wq;
  uint32_t sr, sq;
};

// Starts a stream at reference position pr of `rseq` and query position pq
// of `qseq`, given the first group's words.
__device__ __forceinline__ void stream_begin(Stream &st, const uint8_t *rseq, uint32_t pr, const uint8_t *qseq,
                                             uint32_t pq, uint4 f) {
  st.ra = f.x;
  st.rb = f.y;
  st.qa = f.z;
  st.qb = f.w;
  st.sr = (pr & 3u) * 8u;
  st.sq = (pq & 3u) * 8u;
  st.wr = word_ptr(rseq + pr) + 2;  // the carried word
  st.wq = word_ptr(qseq + pq) + 2;
  st.rc = __ldg(st.wr);
  st.r1 = __ldg(st.wr + 1);
  st.r2 = __ldg(st.wr + 2);
  st.qc = __ldg(st.wq);
  st.q1 = __ldg(st.wq + 1);
  st.q2 = __ldg(st.wq + 2);
}

// The thread-per-hit gate over the warp's tile of nt hits.
template <int TW>
__device__ __forceinline__ void gate_run(const GateArgs &a, const char *subb, WarpTile<TW> &wt, uint32_t nt,
                                         unsigned long long h0, unsigned long long &cells_acc) {
  const uint8_t *ref = a.w.ref, *ref_rev = a.w.ref_rev, *qbuf = a.w.qbuf;
  const int32_t X = a.xdrop;
  const uint32_t lane = threadIdx.x & 31;
  bool have = false, exhausted = false, second = false, capped = false;
  uint32_t t = 0, n = 0, cells = 0, cells_r = 0;
  int32_t S = 0, M = 0, rmax = 0;
  Stream st;
  st.wr = st.wq = nullptr;
  st.ra = st.rb = st.qa = st.qb = st.rc = st.r1 = st.r2 = st.qc = st.q1 = st.q2 = st.sr = st.sq = 0;
  uint32_t cursor = 0;  // next unclaimed hit of the tile (the same in every lane)
  while (true) {
    if (!exhausted) {
      const unsigned need = __ballot_sync(0xffffffffu, !have);
      if (need) {
        const uint32_t base = cursor;
        cursor += (uint32_t)__popc(need);
        if (cursor >= nt) exhausted = true;
        if (!have) {
          const uint32_t mine = base + __popc(need & lanemask_lt());
          if (mine < nt) {
            have = true;
            second = false;
            t = mine;
            const uint32_t nr = wt.hit_n[t] & 0xFFFFu;
            capped = nr > a.cap;
            n = capped ? a.cap : nr;
            S = M = 0;
            cells = 0;
            stream_begin(st, ref, wt.hit_r[t], qbuf, wt.hit_q[t], wt.u.pass.right[t]);
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, have) && exhausted) break;
    if (!have) continue;
    // ---- eight cells ----
    // codes are 0..7, so (r << 5) | (q << 2) is the byte offset of sub[r*8+q]
    const uint32_t ta = (st.ra << 5) | (st.qa << 2), tb = (st.rb << 5) | (st.qb << 2);
    // the next group from the carried and prefetched words
    const uint32_t nra = __funnelshift_r(st.rc, st.r1, st.sr), nrb = __funnelshift_r(st.r1, st.r2, st.sr);
    const uint32_t nqa = __funnelshift_r(st.qc, st.q1, st.sq), nqb = __funnelshift_r(st.q1, st.q2, st.sq);
    const int32_t Ms = M;
    int32_t Si[8];
    int32_t Smin = S;
    HZ_PAIR(ta, 0, 8, 0)
    HZ_PAIR(ta, 16, 24, 2)
    HZ_PAIR(tb, 0, 8, 4)
    HZ_PAIR(tb, 16, 24, 6)
    // first valid cell with M_i - S_i > xdrop, if the bound says there may be one
    const uint32_t v = min(n, 8u);
    uint32_t dm = 0;
    int32_t Mi[8];
    if ((int32_t)((uint32_t)M - (uint32_t)Smin) > X || n <= 8) {
      int32_t m = Ms;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        m = max(m, Si[i]);
        Mi[i] = m;
        dm |= (uint32_t)((int32_t)((uint32_t)m - (uint32_t)Si[i]) > X) << i;
      }
      dm &= (1u << v) - 1u;
    }
    if (!dm && n > 8) {  // no drop and more cells left: advance the stream
      n -= 8;
      cells += 8;
      st.ra = nra;
      st.rb = nrb;
      st.qa = nqa;
      st.qb = nqb;
      st.rc = st.r2;
      st.qc = st.q2;
      st.wr += 2;
      st.wq += 2;
      if (n > 8) {  // words of the group after next (never beyond the padding)
        st.r1 = __ldg(st.wr + 1);
        st.r2 = __ldg(st.wr + 2);
        st.q1 = __ldg(st.wq + 1);
        st.q2 = __ldg(st.wq + 2);
      }
      continue;
    }
    // The extension ends in this group: at the first valid cell with
    // M - S > xdrop (keeping the maximum from before it), or after the v
    // valid cells left before the edge or the cap.
    const uint32_t stop = dm ? (uint32_t)(__ffs(dm) - 1) : v;
    int32_t res = Ms;
#pragma unroll
    for (int i = 1; i <= 8; i++)
      if ((uint32_t)i == stop) res = Mi[i - 1];
    cells += dm ? stop + 1 : v;
    if (!dm && capped) {  // long: the exact kernel redoes the hit; its cells are counted there
      uint32_t at = atomicAdd(&a.tot->cand, 1u);
      if (at < a.cand_cap)
        a.cand[at] = Cand{scope_of(a.scope_lo, min(a.tot->n_scopes, a.scope_cap), h0 + t), wt.hit_r[t],
                          wt.hit_q[t], wt.hit_call[t] | kLongFlag};
      have = false;
    } else if (!second) {  // the right extension ended: start the left one
      rmax = res;
      cells_r = cells;
      second = true;
      const uint32_t nl = wt.hit_n[t] >> 16;
      capped = nl > a.cap;
      n = capped ? a.cap : nl;
      S = M = 0;
      cells = 0;
      stream_begin(st, ref_rev, a.w.rlen - wt.hit_r[t], qbuf, wt.hit_ql[t], wt.u.pass.left[t]);
    } else {
      cells_acc += cells + cells_r;
      int32_t total = (int32_t)((uint32_t)rmax + (uint32_t)res);
      if (sat_i32((double)__int2float_rn(total)) >= a.hspthresh) {
        uint32_t at = atomicAdd(&a.tot->cand, 1u);
        if (at < a.cand_cap)
          a.cand[at] = Cand{scope_of(a.scope_lo, min(a.tot->n_scopes, a.scope_cap), h0 + t), wt.hit_r[t],
                            wt.hit_q[t], wt.hit_call[t]};
      }
      have = false;
    }
  }
}

// Fills the first eight cells of both extensions of every hit of the warp's
// tile.
template <int TW>
__device__ __forceinline__ void prepare_first(const GateArgs &a, WarpTile<TW> &wt, uint32_t nt, uint32_t lane) {
  for (uint32_t i = lane; i < nt; i += 32) {
    const uint32_t r0 = wt.hit_r[i];
    uint32_t ra, rb, qa, qb;
    first_group(a.w.ref, r0, &ra, &rb);
    first_group(a.w.qbuf, wt.hit_q[i], &qa, &qb);
    wt.u.pass.right[i] = make_uint4(ra, rb, qa, qb);
    first_group(a.w.ref_rev, a.w.rlen - r0, &ra, &rb);
    first_group(a.w.qbuf, wt.hit_ql[i], &qa, &qb);
    wt.u.pass.left[i] = make_uint4(ra, rb, qa, qb);
  }
}

// Bucket lookups issued per group of seeds, so their loads are in flight
// together.
constexpr uint32_t kLookupBatch = 4;

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
    __syncwarp();                 // the previous tile's gate is done with the union
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
      wt.hit_ql[i] = cd.qoff_rev + cd.qlen - (q0 - cd.qoff);
      wt.hit_n[i] = min(nr, 0xFFFFu) | (min(nl, 0xFFFFu) << 16);
      wt.hit_call[i] = hc;
    }
    __syncwarp();
    // (3) the score gate, both extensions of a hit by one lane
    prepare_first<TW>(a, wt, nt, lane);
    __syncwarp();
    gate_run<TW>(a, subb, wt, nt, h0, cells_acc);
  }
  for (int d = 16; d > 0; d >>= 1) cells_acc += __shfl_down_sync(0xffffffffu, cells_acc, d);
  if (lane == 0 && cells_acc) atomicAdd(&a.tot->cells, cells_acc);
}

}  // namespace hz
