// Long candidates extended in lockstep (included by hz_wave.cuh after
// hz_gate2.cuh).
//
// A hit whose extension runs past the score gate's cell cap is a "long"
// candidate: the gate stops scoring it and the exact kernel has to redo both
// directions from the anchor (src/gpu/kernels.rs:1279-1406 does this
// warp-wide for every hit).  On repeat-dense input these extensions run to
// hundreds or thousands of cells.  long_kernel extends every long candidate
// of a wave to its end, one lane per candidate-direction, in the gate's
// rounds of kRound cells over the 2-bit packed sequences, and finds in each
// direction the maximum and the first cell that reaches it.  It writes them
// into the candidate and marks it kDoneFlag, so the exact kernel is left
// with the entropy and the accept.
//
// The maximum's position is found without a per-cell test: in a round whose
// cells are all valid the main pass notes the last eight-cell group in which
// the running maximum rose (the first cell reaching the round's final
// maximum lies in it) together with that group's starting sum, and only
// when the direction ends is that one group rescored.  A round that stops
// early (a drop, a special base, the edge) searches its own valid groups at
// once, from the group states it keeps in shared memory and the codes it
// still holds in registers.
//
// Semantics are exact_dir4's: cells counted up to and including the first
// dropping cell (or to the edge); the right position is the cell offset of
// the maximum (-1 when the maximum is the empty extension's 0), the left one
// the offset + 1 (0 then).
#pragma once

namespace hz {

constexpr uint32_t kDoneFlag = 1u << 30;  // Cand::call: maxima and positions filled in by long_kernel

struct LongArgs {
  const uint4 *ref, *refr, *qry, *qryr;  // packed halves (pack2_kernel)
  const uint8_t *ref8, *qry8;            // 8-bit codes of the target and of the query store
  uint32_t rlen, qtotal;
  const CallDev *calls;
  Cand *cand;
  uint32_t cand_cap;
  WaveTotals *tot;
  int32_t sub[64];
  int32_t xdrop;
  uint32_t late_max_safe;  // as GateArgs::late_max_safe
};

struct LongWarp {
  uint32_t queue[64];          // long candidates claimed by the warp, not yet on a lane
  uint32_t grp[kGroups][32];   // group states of a round, as in gate2_kernel
};

struct LongSmem {
  int32_t sub[64];
  int8_t tbl[16];
  LongWarp warp[kGateWarps];
};

// The first of the eight cells whose codes are the low 16 bits of r and q at
// which the running sum, starting from s, equals target (8 if none does).
__device__ __forceinline__ uint32_t first_reach(const int8_t *tbl, uint32_t r, uint32_t q, int32_t s,
                                                int32_t target) {
  uint32_t tw[4];
  pair_words(r & 0xFFFFu, q & 0xFFFFu, tw);
  uint32_t c = 8;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    s = wadd(s, cell_score(tbl, tw, i));
    if (c == 8 && s == target) c = (uint32_t)i;
  }
  return c;
}

__global__ void __launch_bounds__(kGateThreads) long_kernel(LongArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LongSmem &sm = *reinterpret_cast<LongSmem *>(smem_raw);
  if (threadIdx.x < 64) sm.sub[threadIdx.x] = a.sub[threadIdx.x];
  if (threadIdx.x < 16) sm.tbl[threadIdx.x] = (int8_t)a.sub[(threadIdx.x & 3u) * kNuc + (threadIdx.x >> 2)];
  __syncthreads();  // the block's only barrier
  LongWarp &wp = sm.warp[threadIdx.x >> 5];
  const int8_t *tbl = sm.tbl;
  const uint32_t lane = threadIdx.x & 31;
  const int32_t X = a.xdrop;
  const uint32_t ncand = min(a.tot->cand, a.cand_cap);
  unsigned long long cells_acc = 0;
  uint32_t qn = 0;  // candidates in the warp's queue (warp-uniform)
  bool exhausted = false;

  // lane state: the candidate (index, anchors, left edge, call word), the
  // direction, the next round's first base in the direction's packed halves,
  // cells left to the edge, running sum and maximum, cells scored in the
  // direction and in both, the maximum's first cell (-1: none yet) or the
  // group that holds it (pbase >= 0, with the group's starting sum pS), and
  // the right direction's result
  bool have = false;
  uint32_t ci = 0, r0 = 0, q0 = 0, nl = 0, dir = 0, rp = 0, qp = 0, n = 0, cells = 0, tcells = 0;
  int32_t S = 0, M = 0, mpos = -1, pbase = -1, pS = 0, rmax = 0, rpos = -1;
  auto start = [&](uint32_t d, uint32_t edge) {
    dir = d;
    n = edge;
    rp = d ? a.rlen - r0 : r0;
    qp = d ? a.qtotal - q0 : q0;
    S = 0;
    M = 0;
    cells = 0;
    mpos = -1;
    pbase = -1;
  };
  while (true) {
    const unsigned need = __ballot_sync(0xffffffffu, !have);
    if (need && qn < (uint32_t)__popc(need) && !exhausted) {
      // claim chunks of 32 candidates and queue the long ones
      while (qn < 32 && !exhausted) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&a.tot->long_next, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= ncand) {
          exhausted = true;
          break;
        }
        const uint32_t idx = base + lane;
        const bool lg = idx < ncand && (a.cand[idx].call & kLongFlag) != 0;
        const unsigned b = __ballot_sync(0xffffffffu, lg);
        if (lg) wp.queue[qn + (uint32_t)__popc(b & lanemask_lt())] = idx;
        qn += (uint32_t)__popc(b);
      }
      __syncwarp();
    }
    if (need && qn) {
      const uint32_t k = (uint32_t)__popc(need & lanemask_lt());
      if (!have && k < qn) {
        ci = wp.queue[qn - 1 - k];
        const Cand c = a.cand[ci];
        const CallDev cd = a.calls[c.call & ~(kLongFlag | kDoneFlag)];
        r0 = c.r0;
        q0 = c.q0;
        nl = min(r0, q0 - cd.qoff);
        have = true;
        tcells = 0;
        start(0, min(a.rlen - r0, cd.qoff + cd.qlen - q0));
      }
      qn -= min((uint32_t)__popc(need), qn);
      __syncwarp();
    }
    if (!__any_sync(0xffffffffu, have)) {
      if (exhausted && qn == 0) break;
      continue;
    }
    if (!have) n = 0;  // an idle lane scores an empty window at base 0
    const uint32_t prp = have ? rp : 0u, pqp = have ? qp : 0u;
    uint32_t Rc[kChunks], Qc[kChunks], RS0, RS1, QS0, QS1;
    window_round(dir ? a.refr : a.ref, prp, Rc, &RS0, &RS1);
    window_round(dir ? a.qryr : a.qry, pqp, Qc, &QS0, &QS1);
    const uint32_t v = min(n, (uint32_t)kRound);
    const uint32_t sp0 = (RS0 | QS0) & (v >= 32 ? 0xFFFFFFFFu : ((1u << v) - 1u));
    const uint32_t sp1 = (RS1 | QS1) & (v >= 64 ? 0xFFFFFFFFu : v > 32 ? ((1u << (v - 32)) - 1u) : 0u);
    const uint32_t vv = sp0 ? (uint32_t)(__ffs(sp0) - 1) : sp1 ? 32u + (uint32_t)(__ffs(sp1) - 1) : v;

    // the gate's main pass, noting the last group in which the maximum rose
    uint32_t flags = 0;
    int32_t gi = -1;
#pragma unroll
    for (int h = 0; h < kChunks; h++) {
      uint32_t tw[4];
      pair_words(Rc[h], Qc[h], tw);
#pragma unroll
      for (int gg = 0; gg < 2; gg++) {
        const int g = 2 * h + gg;
        wp.grp[g][lane] = __byte_perm((uint32_t)S, (uint32_t)M, 0x5410u);
        const int32_t Mg = M;
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
        gi = M > Mg ? g : gi;
      }
    }
    // exact end of the round, as in gate2_kernel
    const uint32_t gv = vv >> 3;
    uint32_t todo = have ? (flags | (gv < (uint32_t)kGroups ? 1u << gv : 0u)) & ((2u << gv) - 1u) : 0u;
    bool ended = false, dropped = false;
    int32_t res = 0;
    uint32_t used = kRound;
    int32_t Sf = S, Mf = M;
    while (__any_sync(0xffffffffu, todo != 0)) {
      if (todo) {
        const uint32_t g = (uint32_t)(__ffs(todo) - 1);
        todo &= todo - 1;
        const uint32_t st = wp.grp[g][lane];
        int32_t Se = near16(S, st & 0xFFFFu), Me = near16(S, st >> 16);
        const uint32_t ch = g >> 1;
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
          int32_t D = (int32_t)((uint32_t)Me - (uint32_t)Se);
          uint32_t dm = 0;
#pragma unroll
          for (int i = 0; i < 8; i++) {
            D = max((int32_t)((uint32_t)D - (uint32_t)cell_score(tbl, tw, i)), 0);
            dm |= (uint32_t)(D > X) << i;
          }
          if (dm) {
            ended = dropped = true;
            res = g + 1 < (uint32_t)kGroups ? near16(S, wp.grp[g + 1][lane] >> 16) : M;
            used = 8 * g + (uint32_t)(__ffs(dm) - 1) + 1;
            todo = 0;
          }
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
        if (d < 8) {
          ended = dropped = true;
          res = Me;
          used = 8 * g + d + 1;
          todo = 0;
        } else if (g == gv) {
          Sf = Se;
          Mf = Me;
          used = vv;
          todo = 0;
        }
      }
    }
    if (have) {
      bool special_max = false;
      if (!dropped && vv < (uint32_t)kRound && vv < v) {  // a special base at cell vv
        const uint32_t pr = rp + vv, pq = qp + vv;
        const uint32_t r8 = dir ? a.rlen - 1u - pr : pr, q8 = dir ? a.qtotal - 1u - pq : pq;
        const int32_t Sx = wadd(Sf, sm.sub[a.ref8[r8] * kNuc + a.qry8[q8]]);
        const int32_t Mx = max(Mf, Sx);
        used = vv + 1;
        if ((int32_t)((uint32_t)Mx - (uint32_t)Sx) > X) {
          ended = dropped = true;
          res = Mf;
        } else {
          special_max = Sx > Mf;
          Sf = Sx;
          Mf = Mx;
        }
      }
      // where the maximum the round ends with was first reached
      const int32_t Mr = dropped ? res : Mf;
      const int32_t M0 = near16(S, wp.grp[0][lane] >> 16);  // the maximum at the round's start
      if (special_max) {
        mpos = (int32_t)(cells + vv);
        pbase = -1;
      } else if (Mr > M0) {
        if (!dropped && used == (uint32_t)kRound) {  // every group valid: the main pass's last rise
          pbase = (int32_t)(cells + 8u * (uint32_t)gi);
          pS = near16(S, wp.grp[gi][lane] & 0xFFFFu);
        } else {  // the last valid group that starts below Mr holds the first cell reaching it
          uint32_t g = (used - 1) >> 3;
          while (g > 0 && near16(S, wp.grp[g][lane] >> 16) >= Mr) g--;
          static_assert(kChunks == 3, "the chunk select below names three code words");
          const uint32_t hw = (g >> 1) == 0 ? Rc[0] : (g >> 1) == 1 ? Rc[1] : Rc[2];
          const uint32_t qw = (g >> 1) == 0 ? Qc[0] : (g >> 1) == 1 ? Qc[1] : Qc[2];
          const uint32_t sh = (g & 1u) << 4;
          mpos = (int32_t)(cells + 8u * g +
                           first_reach(tbl, hw >> sh, qw >> sh, near16(S, wp.grp[g][lane] & 0xFFFFu), Mr));
          pbase = -1;
        }
      }
      if (!dropped) {
        S = Sf;
        M = Mf;
        if (used >= n) {
          ended = true;
          res = M;
        }
      }
      cells += used;
      rp += used;
      qp += used;
      n -= min(used, n);
    }
    if (ended) {
      if (pbase >= 0) {  // rescore the group noted by the main pass
        const uint32_t at = (uint32_t)pbase - cells;  // negative offset from rp, as uint32 arithmetic
        uint32_t rlo, rhi, rsp, qlo, qhi, qsp;
        window32(dir ? a.refr : a.ref, rp + at, &rlo, &rhi, &rsp);
        window32(dir ? a.qryr : a.qry, qp + at, &qlo, &qhi, &qsp);
        mpos = pbase + (int32_t)first_reach(tbl, rlo, qlo, pS, res);
        pbase = -1;
      }
      tcells += cells;
      if (dir == 0) {
        rmax = res;
        rpos = mpos;
        start(1, nl);
      } else {
        Cand &c = a.cand[ci];
        c.rmax = rmax;
        c.lmax = res;
        c.rpos = rpos;
        c.lpos = mpos + 1;
        c.call |= kDoneFlag;
        cells_acc += tcells;
        have = false;
      }
    }
  }
  for (int d = 16; d > 0; d >>= 1) cells_acc += __shfl_down_sync(0xffffffffu, cells_acc, d);
  if (lane == 0 && cells_acc) atomicAdd(&a.tot->cells, cells_acc);
}

}  // namespace hz
