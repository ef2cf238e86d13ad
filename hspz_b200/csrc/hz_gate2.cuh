// Lockstep score gate over 2-bit packed sequences (included by hz_wave.cuh).
//
// The same work as gate_kernel -- fused hit expansion and the X-drop score
// bound of every hit, src/gpu/kernels.rs:521-1057 -- organised so that a
// warp's 32 lanes run one instruction stream without divergence in the hot
// loop:
//   * a lane owns one hit-direction at a time and scores it in rounds of 48
//     cells (kRound), every lane the same 48 cells' worth of instructions
//     whether its extension ends in the round or not (random hits end after
//     ~23 cells to the right and ~41 to the left, so most directions take one
//     round);
//   * the reference and query are read 2 bits per base (pack2_kernel), so a
//     round's cells are three 16-cell code words per sequence (three 16-byte
//     loads) and
//     a cell's substitution score is one byte extract and one shared-memory
//     byte load from a table indexed by the pair of codes;
//   * a left extension walks the reversed copy of each sequence forwards, so
//     both directions are the same code;
//   * after a round the lanes whose extension ended in it find the exact end
//     cell and the maximum before it by rescoring one eight-cell group, and
//     take the next hit-direction from the warp's tile;
//   * a lane keeps its hit's anchors, call and left edge in registers, so
//     when the tile runs out the warp sets up the next one at once while the
//     lanes still on the old tile's hits carry on -- no lane waits for the
//     slowest hit of a tile.
// Bases that are not uppercase ACGT (soft-masked, N, other, separator) are
// marked in a side mask; a round stops at the first one and that cell is
// scored from the 8-bit codes and the full 8x8 table.
//
// The extension semantics are those of the scalar oracle and the reference
// warp kernel: S += sub[r][q]; M' = max(M, S) includes the cell; the
// extension stops at the first cell with M' - S > xdrop and keeps the maximum
// from before it, or at the edge.  A hit becomes a candidate when
// (i32)(f32)(right max + left max) >= hspthresh, or when a direction runs
// past `cap` cells (then the exact kernel redoes it).
#pragma once

namespace hz {

constexpr int kRound = 48;             // cells a lane scores per round
constexpr int kChunks = kRound / 16;   // 16-cell code words per sequence in a round
constexpr int kGroups = kRound / 8;    // eight-cell groups per round

// The kRound bases of a packed half that start at base p: their codes, 16
// per word, and their special bits (cells 0..31 in *sp_lo, the rest in
// *sp_hi), from the 16-byte records that hold them.
__device__ __forceinline__ void window_round(const uint4 *__restrict__ blk, uint32_t p, uint32_t code[kChunks],
                                             uint32_t *sp_lo, uint32_t *sp_hi) {
  constexpr int kRec = (kRound + 31) / 32 + 1;
  uint4 r[kRec];
#pragma unroll
  for (int i = 0; i < kRec; i++) r[i] = __ldg(blk + (p >> 5) + i);
  uint32_t c[2 * kRec];
#pragma unroll
  for (int i = 0; i < kRec; i++) {
    c[2 * i] = r[i].x;
    c[2 * i + 1] = r[i].y;
  }
  const uint32_t o = p & 31u, sh = (o & 15u) << 1;
  const bool upper = o >= 16;  // the window starts in a record's second code word
  uint32_t cs[kChunks + 1];
#pragma unroll
  for (int k = 0; k <= kChunks; k++) cs[k] = upper ? c[k + 1] : c[k];
#pragma unroll
  for (int k = 0; k < kChunks; k++) code[k] = __funnelshift_r(cs[k], cs[k + 1], sh);
  *sp_lo = __funnelshift_r(r[0].z, r[1].z, o);
  *sp_hi = kRound > 32 ? __funnelshift_r(r[1].z, r[kRec - 1].z, o) : 0u;
}

template <int TW>
struct WarpTile2 {
  uint32_t slot_bst[TW];  // pos_table index of the slot's first in-tile hit
  uint32_t slot_q[TW];    // query anchor (absolute)
  uint32_t slot_call[TW];
  uint32_t hit_slot[TW];  // first hit of the hit's slot + 1 (mark, then max-scan)
  uint32_t hit_r[TW];     // reference anchor
  uint32_t hit_n[TW];     // cells to the right edge | cells to the left edge << 16 (each saturated)
  uint32_t hdr[4];        // the claimed next tile's first position, the position after it, its call
  // each lane's running sum (low half) and maximum (high half) at the start
  // of each group of a round, both modulo 2^16 (near16 restores them)
  uint32_t grp[kGroups][32];
};

template <int TW>
struct Gate2Smem {
  int32_t sub[64];
  int8_t tbl[16];  // score of the pair of ACGT codes: reference code | query code << 2 (see pair_words)
  WarpTile2<TW> warp[kGateWarps];
};

struct Gate2Args {
  GateArgs g;
  // packed sequences (pack2_kernel's records): the forward and the reversed
  // half of the reference and of the query store
  const uint4 *ref, *refr, *qry, *qryr;
  uint32_t qtotal;  // bases of the query store (the reversed query half is it read backwards)
};

// The four index words of 16 cells: word j holds cells j, j+4, j+8, j+12 in
// its bytes 0..3, each byte being that cell's table index (reference code |
// query code << 2) with its upper four bits clear.  Every lane's score lookup
// then falls in the same 16 bytes of shared memory, four banks, so a warp's
// lookup is one wavefront whatever the codes.
__device__ __forceinline__ void pair_words(uint32_t r, uint32_t q, uint32_t t[4]) {
  const uint32_t x = (r & 0x33333333u) | ((q << 2) & 0xCCCCCCCCu);  // nibble n: index of cell 2n
  const uint32_t y = ((r >> 2) & 0x33333333u) | (q & 0xCCCCCCCCu);  // nibble n: index of cell 2n + 1
  t[0] = x & 0x0F0F0F0Fu;
  t[1] = y & 0x0F0F0F0Fu;
  t[2] = (x >> 4) & 0x0F0F0F0Fu;
  t[3] = (y >> 4) & 0x0F0F0F0Fu;
}

// Score of cell k (0..15) of the 16 cells whose index words are t.
__device__ __forceinline__ int32_t cell_score(const int8_t *tbl, const uint32_t t[4], int k) {
  return tbl[__byte_perm(t[k & 3], 0u, 0x4440u + (uint32_t)(k >> 2))];
}

__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }

// The value v with v = h (mod 2^16) and base - 32768 <= v < base + 32768.
// A round's group states are read back against the running sum after all
// its kRound cells, which lies within kRound * 128 of every stored sum; a
// stored maximum read back exceeds its sum by at most xdrop plus one group's
// fall, so every value read lies within kRound * 255 + xdrop of the base
// (gate2_usable checks that this is below 32768).
__device__ __forceinline__ int32_t near16(int32_t base, uint32_t h) {
  return wadd(base, (int32_t)(int16_t)(uint16_t)(h - (uint32_t)base));
}

// 4-byte global -> shared copy that completes asynchronously (no register
// holds the value), and the wait for all of the thread's copies.
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// SPARSE: the setup for targets whose buckets hold few positions, where a
// 128-hit tile spans many query positions (10-20 Mbp bins): a lane per
// position instead of per (position, seed) pair.  The engine picks it from
// the target's average bucket size.
template <int TW, bool SPARSE>
__global__ void __launch_bounds__(kGateThreads, 4) gate2_kernel(Gate2Args a2) {
  static_assert(TW % 32 == 0, "a warp tile is a multiple of 32 hits");
  const GateArgs &a = a2.g;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Gate2Smem<TW> &sm = *reinterpret_cast<Gate2Smem<TW> *>(smem_raw);
  if (a.tot->status & 4u) return;  // no tile table: the host reruns the wave with a larger one
  if (threadIdx.x < 64) sm.sub[threadIdx.x] = a.sub[threadIdx.x];
  if (threadIdx.x < 16) sm.tbl[threadIdx.x] = (int8_t)a.sub[(threadIdx.x & 3u) * kNuc + (threadIdx.x >> 2)];
  __syncthreads();  // the block's only barrier
  WarpTile2<TW> &wt = sm.warp[threadIdx.x >> 5];
  const int8_t *tbl = sm.tbl;
  const uint32_t lane = threadIdx.x & 31;
  const int32_t X = a.xdrop;
  const uint32_t rlen = a.w.rlen, qtotal = a2.qtotal;
  unsigned long long cells_acc = 0;
  const unsigned long long total = a.tot->hits;
  const uint32_t nz = a.tot->nz;
  const WaveIn &w = a.w;

  // the tile the cursor hands hits out of (warp-uniform)
  unsigned long long h0 = 0;
  uint32_t nt = 0, cursor = 0;
  bool tiles_done = false;
  // the next tile's index, claimed from the work queue once half of the
  // current tile is handed out so that its latency is hidden (lane 0 holds it)
  bool claimed = false;
  unsigned long long claim = 0;
  // The tile setup spreads a tile's (position, seed) pairs over the lanes:
  // 32 / per_pos positions per pass, lane l on seed l % per_pos of position
  // l / per_pos, so all bucket bounds of a pass are loaded at once.
  const uint32_t per = w.per_pos, ppi = 32u / per, lpi = lane / per, lvar = lane - lpi * per;
  bool hdr = false;  // the claimed tile's header is on its way into wt.hdr
  // Takes the next tile from the work queue and sets it up: the hits'
  // anchors, edge distances and slots (query anchor, call).  Every lane takes
  // part; lanes busy with an earlier tile's hits hold what they need of them
  // in registers.
  auto next_tile = [&]() {
    unsigned long long j = claim;
    if (!claimed && lane == 0) j = atomicAdd(&a.tot->tiles, 1ull);
    j = __shfl_sync(0xffffffffu, j, 0);
    const bool have_hdr = claimed && hdr;
    claimed = false;
    hdr = false;
    h0 = j * (unsigned long long)TW;
    cursor = 0;
    if (h0 >= total) {
      tiles_done = true;
      nt = 0;
      return;
    }
    nt = (uint32_t)min((unsigned long long)TW, total - h0);
    uint32_t k0, k1, c0;
    if (have_hdr) {
      cp_async_wait_all();
      __syncwarp();
      k0 = wt.hdr[0];
      k1 = wt.hdr[1];
      c0 = wt.hdr[2];
    } else {
      k0 = a.tile_first[j];
      k1 = a.tile_first[j + 1];
      c0 = a.tile_call[j];
    }
    // positions k0 .. kend cover the tile (k1, the next tile's first
    // position, only if its hits start inside this one; the overlap test
    // below sorts that out)
    const uint32_t kend = min(k1, nz - 1);
    const CallDev call0 = w.calls[c0];
    const uint32_t next_off = c0 + 1 < w.ncalls ? w.calls[c0 + 1].pos_off : 0xFFFFFFFFu;
    __syncwarp();  // every lane has read what it needs of the previous tile
    for (uint32_t i = lane; i < nt; i += 32) wt.hit_slot[i] = 0;
    __syncwarp();
    if constexpr (SPARSE) {
      // a lane per position, its seeds' bucket bounds loaded five at a time
      // (more would spill in this register budget)
      for (uint32_t k = k0 + lane; k <= kend; k += 32) {
        const uint32_t p = a.np_pos[k];
        unsigned long long lo = a.np_excl[k];
        uint32_t kmer, qpos, c = c0;
        CallDev cd = call0;
        if (p >= next_off) {  // the tile reaches into a later call
          while (c + 1 < w.ncalls && w.calls[c + 1].pos_off <= p) c++;
          cd = w.calls[c];
        }
        if (a.np_kmer && !w.seeds) {
          kmer = a.np_kmer[k];
          qpos = cd.start + (p - cd.pos_off);
        } else {
          position_seed(w, cd, p, &qpos, &kmer);
        }
        const uint32_t qa = cd.qoff + qpos + w.shape.size;
        constexpr uint32_t kBatch = 5;
        for (uint32_t v0 = 0; v0 < per; v0 += kBatch) {
          uint32_t beg[kBatch], cnt[kBatch];
#pragma unroll
          for (uint32_t u = 0; u < kBatch; u++) {
            cnt[u] = 0;
            beg[u] = 0;
            if (v0 + u < per) cnt[u] = bucket(w, seed_variant(kmer, v0 + u), &beg[u]);
          }
#pragma unroll
          for (uint32_t u = 0; u < kBatch; u++) {
            const unsigned long long hi = lo + cnt[u];
            if (cnt[u] && hi > h0 && lo < h0 + nt) {
              const unsigned long long first = lo > h0 ? lo : h0;
              const uint32_t sl = (uint32_t)(first - h0);
              wt.slot_bst[sl] = beg[u] + (uint32_t)(first - lo);
              wt.slot_q[sl] = qa;
              wt.slot_call[sl] = c;
              wt.hit_slot[sl] = sl + 1;
            }
            lo = hi;
          }
        }
      }
    } else
    for (uint32_t kb = k0; kb <= kend; kb += ppi) {
      const uint32_t k = kb + lpi;
      const bool act = lpi < ppi && k <= kend;
      uint32_t cnt = 0, beg = 0, qa = 0, c = c0;
      unsigned long long lo = 0;
      if (act) {
        const uint32_t p = a.np_pos[k];
        lo = a.np_excl[k];
        uint32_t kmer, qpos;
        CallDev cd = call0;
        if (p >= next_off) {  // the tile reaches into a later call
          while (c + 1 < w.ncalls && w.calls[c + 1].pos_off <= p) c++;
          cd = w.calls[c];
        }
        if (a.np_kmer && !w.seeds) {
          kmer = a.np_kmer[k];
          qpos = cd.start + (p - cd.pos_off);
        } else {
          position_seed(w, cd, p, &qpos, &kmer);
        }
        qa = cd.qoff + qpos + w.shape.size;
        cnt = bucket(w, seed_variant(kmer, lvar), &beg);
      }
      // the position's earlier seeds' hits come first: inclusive scan of the
      // counts over the position's lanes
      uint32_t incl = cnt;
#pragma unroll
      for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t up = __shfl_up_sync(0xffffffffu, incl, d);
        if (lvar >= d) incl += up;
      }
      if (cnt) {
        lo += incl - cnt;
        const unsigned long long hi = lo + cnt;
        if (hi > h0 && lo < h0 + nt) {
          const unsigned long long first = lo > h0 ? lo : h0;
          const uint32_t sl = (uint32_t)(first - h0);
          wt.slot_bst[sl] = beg + (uint32_t)(first - lo);
          wt.slot_q[sl] = qa;
          wt.slot_call[sl] = c;
          wt.hit_slot[sl] = sl + 1;
        }
      }
    }
    __syncwarp();
    {  // inclusive max-scan of the slot marks
      constexpr int PER = TW / 32;
      uint32_t *mark = wt.hit_slot;
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
    __syncwarp();
    {  // each hit's reference anchor and edge distances; a lane's TW / 32
       // pos_table words and calls are loaded before any is used
      constexpr int PER = TW / 32;
      uint32_t r0[PER], q0[PER], qb[PER], qe[PER];
#pragma unroll
      for (int u = 0; u < PER; u++) {
        const uint32_t i = lane + 32u * (uint32_t)u;
        r0[u] = 0;
        q0[u] = qb[u] = qe[u] = 0;
        if (i < nt) {
          const uint32_t s = wt.hit_slot[i] - 1;
          r0[u] = __ldg(w.pos_table + wt.slot_bst[s] + (i - s));
          q0[u] = wt.slot_q[s];
          const CallDev &cd = w.calls[wt.slot_call[s]];
          qb[u] = cd.qoff;
          qe[u] = cd.qoff + cd.qlen;
        }
      }
#pragma unroll
      for (int u = 0; u < PER; u++) {
        const uint32_t i = lane + 32u * (uint32_t)u;
        if (i < nt) {
          const uint32_t r = r0[u] + w.shape.size;
          const uint32_t nr = min(w.rlen - r, qe[u] - q0[u]), nl = min(r, q0[u] - qb[u]);
          wt.hit_r[i] = r;
          wt.hit_n[i] = min(nr, 0xFFFFu) | (min(nl, 0xFFFFu) << 16);
        }
      }
    }
    __syncwarp();
  };

  // lane state: its hit (anchors, call, index in the wave, left edge), the
  // direction (0 right, 1 left), the next round's first base in the
  // direction's packed halves, cells left to the edge or the cap, running sum
  // and maximum, cells scored so far in the direction
  bool have = false, capped = false;
  uint32_t dir = 0, rp = 0, qp = 0, n = 0, cells = 0, rcells = 0;
  uint32_t hr0 = 0, hq0 = 0, hcall = 0, hnl = 0;
  unsigned long long hidx = 0;
  int32_t S = 0, M = 0, rmax = 0;
  // starts direction d of the lane's hit over `edge` cells
  auto start = [&](uint32_t d, uint32_t edge) {
    capped = edge > a.cap;
    n = capped ? a.cap : edge;
    rp = d ? rlen - hr0 : hr0;
    qp = d ? qtotal - hq0 : hq0;
    dir = d;
    S = 0;
    M = 0;
    cells = 0;
  };
  next_tile();
  while (true) {
    if (!claimed && !tiles_done && 2 * cursor >= nt) {
      if (lane == 0) claim = atomicAdd(&a.tot->tiles, 1ull);
      claimed = true;
    } else if (claimed && !hdr) {
      // a round after the claim: the claimed tile's header, copied into
      // shared memory while this round is scored
      const unsigned long long jn = __shfl_sync(0xffffffffu, claim, 0);
      if (jn * (unsigned long long)TW < total && lane < 3)
        cp_async4(&wt.hdr[lane], lane == 0 ? a.tile_first + jn : lane == 1 ? a.tile_first + jn + 1 : a.tile_call + jn);
      cp_async_commit();
      hdr = true;
    }
    unsigned need = __ballot_sync(0xffffffffu, !have);
    if (need && cursor >= nt && !tiles_done) next_tile();
    if (need && cursor < nt) {
      const uint32_t base = cursor;
      cursor += (uint32_t)__popc(need);
      if (!have) {
        const uint32_t t = base + (uint32_t)__popc(need & lanemask_lt());
        if (t < nt) {
          have = true;
          const uint32_t sl = wt.hit_slot[t] - 1, hn = wt.hit_n[t];
          hr0 = wt.hit_r[t];
          hq0 = wt.slot_q[sl];
          hcall = wt.slot_call[sl];
          hnl = hn >> 16;
          hidx = h0 + t;
          start(0, hn & 0xFFFFu);
        }
      }
    }
    if (!__any_sync(0xffffffffu, have)) {
      if (tiles_done) break;
      continue;  // the next tile is set up at the top
    }
    if (!have) n = 0;  // an idle lane scores an empty window at base 0
    const uint32_t prp = have ? rp : 0u, pqp = have ? qp : 0u;
    uint32_t Rc[kChunks], Qc[kChunks], RS0, RS1, QS0, QS1;
    window_round(dir ? a2.refr : a2.ref, prp, Rc, &RS0, &RS1);
    window_round(dir ? a2.qryr : a2.qry, pqp, Qc, &QS0, &QS1);
    // cells scored from the packed codes this round: up to the edge or cap,
    // and before the first special base
    const uint32_t v = min(n, (uint32_t)kRound);
    const uint32_t sp0 = (RS0 | QS0) & (v >= 32 ? 0xFFFFFFFFu : ((1u << v) - 1u));
    const uint32_t sp1 = (RS1 | QS1) & (v >= 64 ? 0xFFFFFFFFu : v > 32 ? ((1u << (v - 32)) - 1u) : 0u);
    const uint32_t vv = sp0 ? (uint32_t)(__ffs(sp0) - 1) : sp1 ? 32u + (uint32_t)(__ffs(sp1) - 1) : v;

    // every lane scores all kRound cells; per eight-cell group it keeps the
    // state before the group (in shared memory) and flags the group when its
    // final maximum minus its smallest sum exceeds xdrop (no flag: no cell of
    // the group dropped)
    uint32_t flags = 0;
#pragma unroll
    for (int h = 0; h < kChunks; h++) {
      uint32_t tw[4];
      pair_words(Rc[h], Qc[h], tw);
#pragma unroll
      for (int gg = 0; gg < 2; gg++) {
        const int g = 2 * h + gg;
        wt.grp[g][lane] = __byte_perm((uint32_t)S, (uint32_t)M, 0x5410u);
        int32_t lo = 0x7FFFFFFF;
#pragma unroll
        for (int i = 0; i < 8; i += 2) {
          const int k = 8 * gg + i;
          const int32_t S1 = wadd(S, cell_score(tbl, tw, k));
          const int32_t S2 = wadd(S1, cell_score(tbl, tw, k + 1));
          M = __vimax3_s32(M, S1, S2);
          lo = __vimin3_s32(lo, S1, S2);
          S = S2;
        }
        flags |= (uint32_t)((int32_t)((uint32_t)M - (uint32_t)lo) > X) << g;
      }
    }
    // the groups to rescore exactly: flagged ones before the group holding
    // the first unscored cell, and that group itself
    const uint32_t gv = vv >> 3;
    uint32_t todo = have ? (flags | (gv < (uint32_t)kGroups ? 1u << gv : 0u)) & ((2u << gv) - 1u) : 0u;
    bool ended = false, dropped = false;
    int32_t res = 0;
    uint32_t used = kRound;
    int32_t Sf = S, Mf = M;  // state after the round's scored cells
    while (__any_sync(0xffffffffu, todo != 0)) {
      if (todo) {
        const uint32_t g = (uint32_t)(__ffs(todo) - 1);
        todo &= todo - 1;
        const uint32_t st = wt.grp[g][lane];
        int32_t Se = near16(S, st & 0xFFFFu), Me = near16(S, st >> 16);
        const uint32_t ch = g >> 1;  // the code word holding the group (constant indices keep Rc, Qc in registers)
        uint32_t hw = Rc[0], qw = Qc[0];
#pragma unroll
        for (int k = 1; k < kChunks; k++)
          if (ch == (uint32_t)k) {
            hw = Rc[k];
            qw = Qc[k];
          }
        const uint32_t sh = (g & 1u) << 4;
        uint32_t tw[4];
        pair_words((hw >> sh) & 0xFFFFu, (qw >> sh) & 0xFFFFu, tw);
        if (a.late_max_safe && g != gv) {
          // A full group.  No cell within seven after a dropping cell can
          // raise the maximum (7 x the largest score <= xdrop), so the
          // maximum before the drop is the group's final one; only the
          // dropping cell is searched, by the drawdown D = M - S.
          int32_t D = (int32_t)((uint32_t)Me - (uint32_t)Se);
          uint32_t dm = 0;
#pragma unroll
          for (int i = 0; i < 8; i++) {
            D = max((int32_t)((uint32_t)D - (uint32_t)cell_score(tbl, tw, i)), 0);
            dm |= (uint32_t)(D > X) << i;
          }
          if (dm) {
            ended = dropped = true;
            res = g + 1 < (uint32_t)kGroups ? near16(S, wt.grp[g + 1][lane] >> 16) : M;
            used = 8 * g + (uint32_t)(__ffs(dm) - 1) + 1;
            todo = 0;
          }  // else the flag was loose: the next flagged group is looked at
          continue;
        }
        const uint32_t lim = g == gv ? vv - 8 * g : 8u;
        uint32_t d = 8;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const int32_t Sx = wadd(Se, cell_score(tbl, tw, i));
          const int32_t Mx = max(Me, Sx);
          if ((uint32_t)i < lim && d == 8) {
            if ((int32_t)((uint32_t)Mx - (uint32_t)Sx) > X) {
              d = (uint32_t)i;
            } else {
              Se = Sx;
              Me = Mx;
            }
          }
        }
        if (d < 8) {  // the first cell past xdrop: the extension ends there
          ended = dropped = true;
          res = Me;
          used = 8 * g + d + 1;
          todo = 0;
        } else if (g == gv) {  // no drop up to the first unscored cell
          Sf = Se;
          Mf = Me;
          used = vv;
          todo = 0;
        }
      }
    }
    if (have && !dropped) {
      if (vv < (uint32_t)kRound && vv < v) {
        // a special base at cell vv: its score from the 8-bit codes
        const uint32_t pr = rp + vv, pq = qp + vv;
        const uint32_t r8 = dir ? rlen - 1u - pr : pr, q8 = dir ? qtotal - 1u - pq : pq;
        const int32_t sc = sm.sub[w.ref[r8] * kNuc + w.qbuf[q8]];
        const int32_t Sx = wadd(Sf, sc);
        const int32_t Mx = max(Mf, Sx);
        used = vv + 1;
        if ((int32_t)((uint32_t)Mx - (uint32_t)Sx) > X) {
          ended = dropped = true;
          res = Mf;
        } else {
          Sf = Sx;
          Mf = Mx;
        }
      }
      if (!dropped) {
        S = Sf;
        M = Mf;
        if (used >= n) {  // reached the edge or the cap
          ended = true;
          res = M;
        }
      }
    }
    if (have) {
      cells += used;
      rp += used;
      qp += used;
      n -= min(used, n);
    }
    if (ended) {
      const bool spill = !dropped && capped;
      if (spill) {
        uint32_t at = atomicAdd(&a.tot->cand, 1u);
        if (at < a.cand_cap)
          a.cand[at] = Cand{scope_of(a.scope_lo, min(a.tot->n_scopes, a.scope_cap), hidx), hr0, hq0,
                            hcall | kLongFlag, 0, 0};
        have = false;  // the exact kernel redoes both directions
      } else if (dir == 0) {
        rmax = res;
        rcells = cells;
        start(1, hnl);
      } else {
        cells_acc += cells + rcells;
        const int32_t tot = wadd(rmax, res);
        if (a.total_exact ? tot >= a.hspthresh : sat_i32((double)__int2float_rn(tot)) >= a.hspthresh) {
          uint32_t at = atomicAdd(&a.tot->cand, 1u);
          if (at < a.cand_cap)
            a.cand[at] = Cand{scope_of(a.scope_lo, min(a.tot->n_scopes, a.scope_cap), hidx), hr0, hq0, hcall,
                              rmax, res};
        }
        have = false;
      }
    }
  }
  for (int d = 16; d > 0; d >>= 1) cells_acc += __shfl_down_sync(0xffffffffu, cells_acc, d);
  if (lane == 0 && cells_acc) atomicAdd(&a.tot->cells, cells_acc);
}

}  // namespace hz
