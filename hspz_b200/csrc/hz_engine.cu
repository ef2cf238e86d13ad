// Host side of the B200 seed-and-filter engine and its C ABI
// (include/hspz_b200.h).  One engine = one device, one stream, a resident
// target (reference codes, index_table, pos_table), a resident query store
// and two seed slots, mirroring the reference's Engine (src/gpu/mod.rs:817-2307).
//
// Every seed_and_filter call goes through the same wave pipeline
// (hz_wave.cuh).  The plain per-chunk form runs one call per wave and reads
// its HSPs back after each call, as the reference does; the batched form runs
// many calls per wave with one read-back per wave.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>
#include <string>
#include <vector>

#include <cuda.h>

#include "../../include/hspz_b200.h"
#include "hz_kernels.cuh"
#include "hz_scan.cuh"
#include "hz_wave.cuh"
#include "hz_dedup.cuh"

using namespace hz;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(x)                                                                                  \
  do {                                                                                         \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess)                                                                     \
      return fail(e_ == cudaErrorMemoryAllocation ? HZ_E_OOM : HZ_E_CUDA, "%s: %s (%s:%d)", #x, \
                  cudaGetErrorString(e_), __FILE__, __LINE__);                                 \
  } while (0)

#define TRY(x)                  \
  do {                          \
    int r_ = (x);               \
    if (r_ != HZ_OK) return r_; \
  } while (0)

constexpr size_t kPad = 64;  // bytes of padding before and after every sequence buffer
constexpr uint64_t kKeepBuildScratch = 2ull << 30;  // seed table build memory kept for the next build

// Grow-only device buffer.  Growing waits for the stream, because a queued
// kernel may still read the old allocation.
template <typename T> struct DBuf {
  T *p = nullptr;
  size_t cap = 0;
  int ensure(size_t n, cudaStream_t s) {
    if (n <= cap && p) return HZ_OK;
    size_t want = std::max(n, cap + cap / 2);
    if (want == 0) want = 1;
    if (p) {
      CK(cudaStreamSynchronize(s));
      CK(cudaFree(p));
      p = nullptr;
      cap = 0;
    }
    CK(cudaMalloc(&p, want * sizeof(T) + 64));
    cap = want;
    return HZ_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Pinned host buffer, grow-only.
template <typename T> struct HBuf {
  T *p = nullptr;
  size_t cap = 0;
  int ensure(size_t n) {
    if (n <= cap && p) return HZ_OK;
    size_t want = std::max(n, cap + cap / 2);
    if (want == 0) want = 1;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    CK(cudaMallocHost(&p, want * sizeof(T) + 64));
    cap = want;
    return HZ_OK;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

// A sequence buffer with kPad zero bytes on both sides (word loads of the
// extension kernels may touch them; their cells are never scored).
struct SeqBuf {
  DBuf<uint8_t> buf;
  size_t len = 0;
  uint8_t *base() const { return buf.p + kPad; }
  int ensure(size_t n, cudaStream_t s) {
    TRY(buf.ensure(n + 2 * kPad, s));
    CK(cudaMemsetAsync(buf.p, 0, kPad, s));
    CK(cudaMemsetAsync(buf.p + kPad + n, 0, kPad, s));
    len = n;
    return HZ_OK;
  }
};

// --- alphabet tables (src/sequence.rs:66-86) --------------------------------
uint8_t enc_of(uint8_t c) {
  switch (c) {
    case 'A': return 0;
    case 'C': return 1;
    case 'G': return 2;
    case 'T': return 3;
    case 'a': case 'c': case 'g': case 't': return 4;
    case 'n': case 'N': return 5;
    case '&': return 7;
    default: return 6;
  }
}
const char kRevComp[129] =
    "NNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNN"
    "NNNNNN&NNNNNNNNNNNNNNNNNNNNNNNNN"
    "NTVGHNNCDNNMNKNNNNYSAABWNRNNNNNN"
    "NtvghnncdnnmnknnnnysaabwnrnNNNNN";

// --- Shape::parse (src/seed.rs:49-79) ------------------------------------------
int parse_shape(const char *spec, ShapeDev *sh) {
  const char *pat = spec;
  if (!strcmp(spec, "12of19")) pat = "TTT0T00TT00T0T0TTTT";
  else if (!strcmp(spec, "14of22")) pat = "TTT0T0TT00TT00T0T0TTTT";
  memset(sh, 0, sizeof(*sh));
  uint32_t n = 0, k = 0;
  for (const char *c = pat; *c; c++, n++) {
    if (*c == '1' || *c == 'T') {
      if (k >= (uint32_t)kMaxCare) return fail(HZ_E_INVALID, "seed %s has too many care positions", spec);
      sh->pos[k++] = n;
    }
  }
  if (k < 4 || k > 15)
    return fail(HZ_E_INVALID, "seed %s has %u care positions; the seed table requires 4..=15", spec, k);
  sh->size = n;
  sh->kmer_size = k;
  static const uint32_t k12of19[12] = {0, 1, 2, 4, 7, 8, 11, 13, 15, 16, 17, 18};
  sh->is_12of19 = n == 19 && k == 12 && !memcmp(sh->pos, k12of19, sizeof(k12of19));
  for (uint32_t t = 0; t < k; t++) {
    if (t && sh->pos[t] == sh->pos[t - 1] + 1) {
      sh->run_len[sh->nruns - 1]++;
    } else {
      sh->run_start[sh->nruns] = sh->pos[t];
      sh->run_len[sh->nruns] = 1;
      sh->nruns++;
    }
  }
  return HZ_OK;
}

// --- dedup_and_order (src/hsp.rs:62-126) --------------------------------------
// by_diagonal: diagonal, ref_start, len ascending, score descending;
// by_lastz: query_start, ref_start, len ascending, score descending.
inline uint32_t diag_of(const hz_segment_pair &h) { return h.ref_start - h.query_start; }
bool contained(const hz_segment_pair &x, const hz_segment_pair &y) {
  uint32_t xe = x.ref_start + x.len, ye = y.ref_start + y.len;
  return diag_of(x) == diag_of(y) &&
         ((x.ref_start >= y.ref_start && xe <= ye) || (y.ref_start >= x.ref_start && ye <= xe));
}
// Both orders are total over the four fields, so any sort reproduces the
// reference's stable sorts exactly.  Each record is sorted as one 128-bit key
// whose unsigned order is the comparator's (score flipped for descending);
// the record is recovered from the key, since the fields determine it.
typedef unsigned __int128 u128;
inline uint32_t score_desc(int32_t s) { return ~((uint32_t)s ^ 0x80000000u); }
inline int32_t score_of(uint32_t k) { return (int32_t)(~k ^ 0x80000000u); }
inline u128 key4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  return ((u128)a << 96) | ((u128)b << 64) | ((u128)c << 32) | (u128)d;
}
size_t dedup_and_order(hz_segment_pair *h, size_t n) {
  if (n == 0) return 0;
  std::vector<u128> key(n);
  for (size_t i = 0; i < n; i++) key[i] = key4(diag_of(h[i]), h[i].ref_start, h[i].len, score_desc(h[i].score));
  std::sort(key.begin(), key.end());  // by_diagonal
  auto rec = [](u128 k) {
    hz_segment_pair r;
    uint32_t diag = (uint32_t)(k >> 96);
    r.ref_start = (uint32_t)(k >> 64);
    r.query_start = r.ref_start - diag;
    r.len = (uint32_t)(k >> 32);
    r.score = score_of((uint32_t)k);
    return r;
  };
  size_t m = 1;
  hz_segment_pair prev = rec(key[0]);
  key[0] = key4(prev.query_start, prev.ref_start, prev.len, score_desc(prev.score));
  for (size_t i = 1; i < n; i++) {
    hz_segment_pair cur = rec(key[i]);
    if (!contained(prev, cur)) key[m++] = key4(cur.query_start, cur.ref_start, cur.len, score_desc(cur.score));
    prev = cur;
  }
  std::sort(key.begin(), key.begin() + m);  // by_lastz
  for (size_t i = 0; i < m; i++) {
    u128 k = key[i];
    h[i].query_start = (uint32_t)(k >> 96);
    h[i].ref_start = (uint32_t)(k >> 64);
    h[i].len = (uint32_t)(k >> 32);
    h[i].score = score_of((uint32_t)k);
  }
  return m;
}

unsigned grid_for(uint64_t n, unsigned threads, unsigned cap = 148u * 64u) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return (unsigned)std::min<uint64_t>(b, cap);
}

}  // namespace

// A sequence packed 2 bits per base for the lockstep gate (pack2_kernel):
// the forward half and the reversed half, each `half` bases, codes and
// special masks.
struct Packed {
  DBuf<uint4> blk;  // one 16-byte record per 32 bases
  uint64_t half = 0;
  bool valid = false;
  const uint4 *half_ptr(int rev) const { return blk.p + (rev ? half / 32 : 0); }
  void release() {
    blk.release();
    valid = false;
  }
};

// ---------------------------------------------------------------------------

// One call as the host sees it: a WGA chunk [start, end) of one strand of one
// staged query, tagged with its LASTZ interval.
struct HostCall {
  uint32_t query;
  uint32_t interval;
  uint32_t strand;  // 0 forward, 1 reverse complement
  uint32_t start, end;
};

// A staged query block: forward and reverse-complement codes in the store.
struct StagedQuery {
  uint32_t off_f = 0, off_r = 0, len = 0;
};

struct Slot {
  int kind = 0;  // 0 empty, 1 uploaded seeds, 2 generated range
  DBuf<uint64_t> seeds;
  uint64_t n = 0;
  int rev = 0;
  uint32_t start = 0, end = 0;
  int transitions = 1;
};

struct ProfEntry {
  double ms = 0;
  uint64_t n = 0;
};

// One output record of a wave: the call and the HSP (after per-scope dedup).
struct WaveRecord {
  uint32_t call;
  hz_segment_pair h;
};

struct Server;
uint64_t server_launches(Server *s);  // kernel launches of a serving loop's workers

struct hz_engine {
  int device = 0;
  int sm_count = 148;
  cudaStream_t st = nullptr;
  cudaStream_t own_st = nullptr;
  hz_config cfg;
  ShapeDev shape;
  uint32_t max_hits = 0;
  // target
  SeqBuf ref;
  uint32_t rlen = 0;
  DBuf<uint32_t> index_table;
  uint64_t index_len = 0;
  DBuf<uint32_t> pos_table;
  uint64_t n_pos = 0;
  // per k-mer: hits of its exact seed and all its transition seeds, capped
  // per seed (the hit count of a query position with that k-mer)
  DBuf<uint32_t> nbr_hits;
  bool has_nbr = false;
  // working memory of the on-device seed table build, kept between builds
  // of up to kKeepBuildScratch bytes (per-bin loads reuse it)
  struct BuildScratch {
    DBuf<uint8_t> ascii, junk;
    DBuf<uint32_t> kmers, flags, keys, vals, keys2, vals2, partial, total, hist, hpartial, excl, ipart;
    uint64_t bytes() const {
      return ascii.cap + junk.cap +
             4 * (kmers.cap + flags.cap + keys.cap + vals.cap + keys2.cap + vals2.cap + partial.cap + total.cap +
                  hist.cap + hpartial.cap + excl.cap + ipart.cap);
    }
    void release() {
      ascii.release();
      junk.release();
      for (auto *b : {&kmers, &flags, &keys, &vals, &keys2, &vals2, &partial, &total, &hist, &hpartial, &excl, &ipart})
        b->release();
    }
  } build;
  Packed ref_p;  // the reference packed for the lockstep gate
  bool has_target = false;
  bool owns_target = true;         // false for serving workers that share the owner's tables
  bool aliases_query = false;      // true for the plain form's extra workspaces (see run_pass_multi)
  std::vector<hz_engine *> twins;  // those workspaces, made on first use
  int plain_streams = 4;           // workspaces (host threads and streams) of a plain pass, 1..4
  struct Server *server = nullptr;  // the serving loop, while one runs
  // query store
  SeqBuf qstore;
  Packed qry_p;  // the query store packed for the lockstep gate
  DBuf<uint8_t> qascii;
  std::vector<StagedQuery> queries;
  uint32_t cur_query = 0;  // the query the per-call entry points work on
  bool has_query = false;
  Slot slot[2];
  // wave buffers
  DBuf<CallDev> calls;
  DBuf<uint32_t> pos_hits, np_pos, call_nz_lo, scope_call, raw_scope, tile_first, tile_call;
  DBuf<uint32_t> pos_kmer, np_kmer;  // k-mer of every seed position, and of every position with hits
  uint32_t tile_cap = 1u << 23;  // entries of the gate's tile table (grows when a wave needs more)
  DBuf<unsigned long long> np_excl, call_hit_lo, scope_lo;
  DBuf<HitNz> np_partial, np_grand;
  DBuf<WaveTotals> tot;
  DBuf<Cand> cand;
  DBuf<SegmentPair> raw;
  HBuf<CallDev> h_calls;
  HBuf<WaveTotals> h_tot;
  HBuf<hz_segment_pair> h_raw;
  HBuf<uint32_t> h_raw_scope, h_scope_call;
  // device dedup of the batched form
  bool device_dedup = true;
  uint32_t device_dedup_min = 1u << 16;  // raw HSPs from which a per-call wave dedups on the device
  DBuf<uint32_t> d_perm_a, d_perm_b, d_keys_a, d_keys_b, d_keep, d_keep_excl, d_hist, d_hpart, d_total;
  DBuf<ScopedHspOut> d_out;
  HBuf<ScopedHspOut> h_out;
  uint32_t cand_cap = 1u << 20, raw_cap = 1u << 20, scope_cap = 0;
  // tuning
  int gate_version = 2;  // 2: lockstep gate over packed sequences (when the scores allow), 1: lane-refill gate
  // hz_run_batched's records, kept between calls so that repeated passes
  // reuse the host memory instead of growing (and faulting in) a new vector
  std::vector<WaveRecord> batch_recs;
  int gate_sparse = -1;  // lockstep gate tile setup: -1 chosen from the target's buckets, 0 pairs, 1 lane per position
  int gate_tile = 128;  // hits per gate warp tile
  uint32_t gate_cap = 128;  // the autotuner's usual choice
  int gate_blocks_per_sm = 0;
  uint64_t wave_positions = 1ull << 27;  // seed positions per batched wave
  uint64_t wave_hits_cap = 1ull << 33;    // hits per batched wave of several calls (tile table <= 512 MB)
  // CUDA graph of the batched wave chain
  bool use_graph = false;
  bool capturing = false;  // a wave chain is being captured on `st`
  cudaGraphExec_t wave_exec = nullptr;
  uint64_t graph_instantiations = 0, graph_updates = 0, graph_launches = 0;
  // profiling
  bool profiling = false;
  struct PendingEvents {
    std::string name;
    cudaEvent_t a, b;
    bool pooled;  // false: the pair belongs to the captured graph
  };
  std::vector<PendingEvents> pending;
  std::vector<cudaEvent_t> event_pool;
  std::map<std::string, std::pair<cudaEvent_t, cudaEvent_t>> graph_events;
  std::map<std::string, ProfEntry> prof;
  std::vector<std::string> prof_order;
  uint64_t launches = 0;
  uint64_t cand_seen = 0;  // gate candidates of every finished wave (serving admission learns from it)

  cudaEvent_t get_event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  // Brackets one launch (or launch group counted as `count` kernels) with
  // events when profiling.
  // While a wave is captured the pair becomes event-record nodes of the
  // graph (one fixed pair per name, read after each graph launch).
  template <typename F> int launch(const char *name, F &&f, int count = 1) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (profiling) {
      if (capturing) {
        auto &ge = graph_events[name];
        if (!ge.first) {
          cudaEventCreate(&ge.first);
          cudaEventCreate(&ge.second);
        }
        a = ge.first;
        b = ge.second;
        cudaEventRecordWithFlags(a, st, cudaEventRecordExternal);
      } else {
        a = get_event();
        b = get_event();
        cudaEventRecord(a, st);
      }
    }
    f();
    launches += count;
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return fail(HZ_E_CUDA, "launch %s: %s", name, cudaGetErrorString(err));
    if (profiling) {
      if (capturing) cudaEventRecordWithFlags(b, st, cudaEventRecordExternal);
      else cudaEventRecord(b, st);
      pending.push_back({name, a, b, !capturing});
    }
    return HZ_OK;
  }
  // Waits for the stream and folds finished event pairs into the profile.
  int sync() {
    CK(cudaStreamSynchronize(st));
    for (auto &pe : pending) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, pe.a, pe.b) == cudaSuccess) {
        if (!prof.count(pe.name)) prof_order.push_back(pe.name);
        prof[pe.name].ms += ms;
        prof[pe.name].n += 1;
      } else {
        cudaGetLastError();  // a pair whose graph never ran
      }
      if (pe.pooled) {
        event_pool.push_back(pe.a);
        event_pool.push_back(pe.b);
      }
    }
    pending.clear();
    return HZ_OK;
  }
  uint32_t per_pos(int transitions) const { return transitions ? 1 + shape.kmer_size : 1; }
};

namespace {

int set_device(hz_engine *e) {
  CK(cudaSetDevice(e->device));
  return HZ_OK;
}

template <int TW> size_t gate_smem() { return sizeof(GateSmem<TW>); }

// Packs n device codes for the lockstep gate (forward and reversed halves).
int pack_seq(hz_engine *e, const uint8_t *codes, uint64_t n, Packed *p) {
  cudaStream_t s = e->st;
  p->valid = false;
  p->half = (n + 64 + 31) & ~31ull;
  const uint64_t blocks = 2 * p->half / 32;
  TRY(p->blk.ensure(blocks + 4, s));
  CK(cudaMemsetAsync(p->blk.p + blocks, 0, 4 * sizeof(uint4), s));  // read by windows past the end
  uint4 *bk = p->blk.p;
  const uint64_t half = p->half;
  TRY(e->launch("pack", [&] { pack2_kernel<<<grid_for(blocks, 256), 256, 0, s>>>(codes, n, half, bk); }));
  p->valid = true;
  return HZ_OK;
}

// The lockstep gate reads each cell's score as a signed byte and keeps
// positions in 32 bits; otherwise the lane-refill gate runs.
bool gate2_usable(const hz_engine *e) {
  if (e->gate_version != 2 || !e->ref_p.valid || !e->qry_p.valid) return false;
  if ((uint64_t)e->rlen + 128 >= (1ull << 32) || (uint64_t)e->qstore.len + 128 >= (1ull << 32)) return false;
  for (int r = 0; r < 4; r++)
    for (int q = 0; q < 4; q++) {
      const int32_t v = e->cfg.sub_mat[r * kNuc + q];
      if (v < -128 || v > 127) return false;
    }
  // the group states a round keeps modulo 2^16 (gate2_kernel, near16)
  return (int64_t)e->cfg.xdrop + kRound * 255 < 32768;
}

template <int TW> size_t gate2_smem() { return sizeof(Gate2Smem<TW>); }

template <int TW, bool SPARSE> int launch_gate2_as(hz_engine *e, const GateArgs &ga) {
  static bool configured[64] = {false};
  static std::mutex mu;  // serving workers launch from several host threads
  size_t smem = gate2_smem<TW>();
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!configured[e->device & 63]) {
      CK(cudaFuncSetAttribute(gate2_kernel<TW, SPARSE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      configured[e->device & 63] = true;
    }
  }
  int per_sm = e->gate_blocks_per_sm;
  if (per_sm <= 0) {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gate2_kernel<TW, SPARSE>, kGateThreads, smem));
    if (per_sm < 1) per_sm = 1;
  }
  Gate2Args a2;
  a2.g = ga;
  a2.ref = e->ref_p.half_ptr(0);
  a2.refr = e->ref_p.half_ptr(1);
  a2.qry = e->qry_p.half_ptr(0);
  a2.qryr = e->qry_p.half_ptr(1);
  a2.qtotal = (uint32_t)e->qstore.len;
  unsigned grid = (unsigned)(e->sm_count * per_sm);
  return e->launch("gate", [&] { gate2_kernel<TW, SPARSE><<<grid, kGateThreads, smem, e->st>>>(a2); });
}

// The sparse tile setup when a tile is expected to span more than three
// passes of (position, seed) pairs (32 / per_pos positions each), from the
// hits per query position: seeds per position times the average bucket.
template <int TW> int launch_gate2(hz_engine *e, const GateArgs &ga) {
  const double per_bucket = (double)e->n_pos / (double)(1ull << (2 * e->shape.kmer_size));
  const double hits_per_pos = std::max(ga.w.per_pos * per_bucket, 1e-9);
  const double positions_per_pass = (double)(32 / ga.w.per_pos);
  const bool sparse =
      e->gate_sparse >= 0 ? e->gate_sparse == 1 : (double)TW / hits_per_pos > 3.0 * positions_per_pass;
  return sparse ? launch_gate2_as<TW, true>(e, ga) : launch_gate2_as<TW, false>(e, ga);
}

// The long candidates of a wave, extended to their ends in lockstep over the
// packed sequences (long_kernel); runs only where the packed gate runs.
int launch_long(hz_engine *e, const GateArgs &ga) {
  static bool configured[64] = {false};
  static std::mutex mu;
  const size_t smem = sizeof(LongSmem);
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!configured[e->device & 63]) {
      CK(cudaFuncSetAttribute(long_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      configured[e->device & 63] = true;
    }
  }
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, long_kernel, kGateThreads, smem));
  if (per_sm < 1) per_sm = 1;
  LongArgs la;
  la.ref = e->ref_p.half_ptr(0);
  la.refr = e->ref_p.half_ptr(1);
  la.qry = e->qry_p.half_ptr(0);
  la.qryr = e->qry_p.half_ptr(1);
  la.ref8 = ga.w.ref;
  la.qry8 = ga.w.qbuf;
  la.rlen = ga.w.rlen;
  la.qtotal = (uint32_t)e->qstore.len;
  la.calls = ga.w.calls;
  la.cand = ga.cand;
  la.cand_cap = ga.cand_cap;
  la.tot = ga.tot;
  memcpy(la.sub, ga.sub, sizeof(la.sub));
  la.xdrop = ga.xdrop;
  la.late_max_safe = ga.late_max_safe;
  const unsigned grid = (unsigned)(e->sm_count * per_sm);
  return e->launch("long", [&] { long_kernel<<<grid, kGateThreads, smem, e->st>>>(la); });
}

template <int TW> int launch_gate(hz_engine *e, const GateArgs &ga) {
  static bool configured[64] = {false};
  static std::mutex mu;  // serving workers launch from several host threads
  size_t smem = gate_smem<TW>();
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!configured[e->device & 63]) {
      CK(cudaFuncSetAttribute(gate_kernel<TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      configured[e->device & 63] = true;
    }
  }
  int per_sm = e->gate_blocks_per_sm;
  if (per_sm <= 0) {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gate_kernel<TW>, kGateThreads, smem));
    if (per_sm < 1) per_sm = 1;
  }
  unsigned grid = (unsigned)(e->sm_count * per_sm);
  return e->launch("gate", [&] { gate_kernel<TW><<<grid, kGateThreads, smem, e->st>>>(ga); });
}

// run_wave's answer for a wave of several calls that holds too many hits:
// nothing was kept, and the caller reruns the calls in smaller waves.
constexpr int kSplitWave = 1;

// Runs calls[0..n) as one wave and appends its deduped HSPs, in call order
// and LASTZ order within each MAX_HITS scope, to *out.  `seeds` (device) is
// the uploaded seed array of a single-call wave, or null.
// dedup_and_order of every scope of a wave on the device (hz_dedup.cuh);
// appends the kept HSPs, in scope order and LASTZ order within each scope.
int dedup_on_device(hz_engine *e, uint32_t nraw, uint32_t n_scopes, uint32_t call_base, std::vector<WaveRecord> *out,
                    hz_stats *st) {
  cudaStream_t s = e->st;
  TRY(e->d_perm_a.ensure(nraw, s));
  TRY(e->d_perm_b.ensure(nraw, s));
  TRY(e->d_keys_a.ensure(nraw, s));
  TRY(e->d_keys_b.ensure(nraw, s));
  TRY(e->d_keep.ensure(nraw, s));
  TRY(e->d_keep_excl.ensure(nraw, s));
  uint64_t rtiles = (nraw + kRadixTile - 1) / kRadixTile;
  TRY(e->d_hist.ensure(rtiles * kRadixBins, s));
  TRY(e->d_hpart.ensure(scan_tiles(std::max<uint64_t>(rtiles * kRadixBins, nraw)) + 1, s));
  TRY(e->d_total.ensure(1, s));
  const unsigned g = grid_for(nraw, 256);
  TRY(e->launch("dedup", [&] { iota_kernel<<<g, 256, 0, s>>>(e->d_perm_a.p, nraw); }));
  uint32_t scope_bytes = 1;
  while (scope_bytes < 4 && (n_scopes >> (8 * scope_bytes))) scope_bytes++;
  // stable LSD passes over the fields of a key, least significant first
  auto sort_by = [&](const int *fields, int nf, uint32_t cnt) -> int {
    uint64_t tiles = (cnt + kRadixTile - 1) / kRadixTile;
    for (int fi = 0; fi < nf; fi++) {
      int f = fields[fi];
      TRY(e->launch("dedup", [&] {
        gather_key_kernel<<<grid_for(cnt, 256), 256, 0, s>>>(e->raw.p, e->raw_scope.p, e->d_perm_a.p, cnt, f,
                                                            e->d_keys_a.p);
      }));
      int passes = f == kScope ? (int)scope_bytes : 4;
      for (int p = 0; p < passes; p++) {
        int shift = 8 * p;
        TRY(e->launch("dedup", [&] {
          radix_hist_kernel<<<(unsigned)tiles, kRadixThreads, 0, s>>>(e->d_keys_a.p, cnt, shift, e->d_hist.p, tiles);
          exclusive_scan<uint32_t>(e->d_hist.p, e->d_hist.p, tiles * kRadixBins, e->d_hpart.p, e->d_total.p, s);
          radix_scatter_kernel<<<(unsigned)tiles, kRadixThreads, 0, s>>>(e->d_keys_a.p, e->d_perm_a.p, cnt, shift,
                                                                        e->d_hist.p, tiles, e->d_keys_b.p,
                                                                        e->d_perm_b.p);
        }, 5));
        std::swap(e->d_keys_a, e->d_keys_b);
        std::swap(e->d_perm_a, e->d_perm_b);
      }
    }
    return HZ_OK;
  };
  static const int by_diagonal_key[5] = {kScoreDesc, kLen, kRefStart, kDiag, kScope};
  static const int by_lastz_key[5] = {kScoreDesc, kLen, kRefStart, kQueryStart, kScope};
  TRY(sort_by(by_diagonal_key, 5, nraw));
  TRY(e->launch("dedup", [&] {
    keep_flag_kernel<<<g, 256, 0, s>>>(e->raw.p, e->raw_scope.p, e->d_perm_a.p, nraw, e->d_keep.p);
    exclusive_scan<uint32_t>(e->d_keep.p, e->d_keep_excl.p, nraw, e->d_hpart.p, e->d_total.p, s);
    compact_perm_kernel<<<g, 256, 0, s>>>(e->d_perm_a.p, e->d_keep_excl.p, e->d_keep.p, nraw, e->d_perm_b.p);
  }, 5));
  uint32_t kept = 0;
  CK(cudaMemcpyAsync(&kept, e->d_total.p, 4, cudaMemcpyDeviceToHost, s));
  TRY(e->sync());
  std::swap(e->d_perm_a, e->d_perm_b);
  TRY(sort_by(by_lastz_key, 5, kept));
  TRY(e->d_out.ensure(kept + 1, s));
  TRY(e->h_out.ensure(kept + 1));
  TRY(e->h_scope_call.ensure(n_scopes + 1));
  TRY(e->launch("dedup", [&] {
    emit_scoped_kernel<<<grid_for(kept, 256), 256, 0, s>>>(e->raw.p, e->raw_scope.p, e->d_perm_a.p, kept, e->d_out.p);
  }));
  CK(cudaMemcpyAsync(e->h_out.p, e->d_out.p, (size_t)kept * sizeof(ScopedHspOut), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(e->h_scope_call.p, e->scope_call.p, (size_t)n_scopes * 4, cudaMemcpyDeviceToHost, s));
  TRY(e->sync());
  for (uint32_t i = 0; i < kept; i++) {
    const ScopedHspOut &r = e->h_out.p[i];
    out->push_back(WaveRecord{e->h_scope_call.p[r.scope] + call_base,
                              hz_segment_pair{r.h.ref_start, r.h.query_start, r.h.len, r.h.score}});
  }
  if (st) st->hsps += kept;
  return HZ_OK;
}

// Captures `chain` (stream work on e->st) into a graph and launches it,
// updating the engine's instantiated graph in place when the new capture has
// the same shape (the usual case: waves differ only in sizes and pointers).
template <typename F> int run_captured(hz_engine *e, F &&chain) {
  cudaStream_t s = e->st;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  e->capturing = true;
  int rc = chain();
  e->capturing = false;
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (rc != HZ_OK || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    e->pending.erase(std::remove_if(e->pending.begin(), e->pending.end(), [](const hz_engine::PendingEvents &p) {
                       return !p.pooled;
                     }),
                     e->pending.end());
    return rc != HZ_OK ? rc : fail(HZ_E_CUDA, "wave capture: %s", cudaGetErrorString(ce));
  }
  if (e->wave_exec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(e->wave_exec, g, &info) == cudaSuccess) {
      e->graph_updates++;
    } else {
      cudaGetLastError();
      cudaGraphExecDestroy(e->wave_exec);
      e->wave_exec = nullptr;
    }
  }
  if (!e->wave_exec) {
    cudaError_t ie = cudaGraphInstantiate(&e->wave_exec, g, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(g);
      e->wave_exec = nullptr;
      return fail(HZ_E_CUDA, "wave graph instantiate: %s", cudaGetErrorString(ie));
    }
    e->graph_instantiations++;
  }
  cudaGraphDestroy(g);
  CK(cudaGraphLaunch(e->wave_exec, s));
  e->graph_launches++;
  return HZ_OK;
}

// The host side of a wave's dedup: the wave's raw HSPs and their scopes,
// already read back into e->h_raw / h_raw_scope / h_scope_call, are grouped by
// scope and deduped per scope; the records go to *out in scope order, with
// their wave-relative call index plus `call_base`.
void host_dedup(hz_engine *e, uint32_t nraw, uint32_t n_scopes, uint32_t call_base, std::vector<WaveRecord> *out,
                hz_stats *st) {
  // counting sort by scope
  std::vector<uint32_t> start(n_scopes + 1, 0);
  for (uint32_t i = 0; i < nraw; i++) start[e->h_raw_scope.p[i] + 1]++;
  for (uint32_t k = 0; k < n_scopes; k++) start[k + 1] += start[k];
  std::vector<hz_segment_pair> sorted(nraw);
  std::vector<uint32_t> cur(start.begin(), start.end() - 1);
  for (uint32_t i = 0; i < nraw; i++) sorted[cur[e->h_raw_scope.p[i]]++] = e->h_raw.p[i];
  for (uint32_t k = 0; k < n_scopes; k++) {
    size_t a = start[k], b = start[k + 1];
    if (a == b) continue;
    size_t kept = dedup_and_order(sorted.data() + a, b - a);
    if (st) st->hsps += kept;
    uint32_t c = e->h_scope_call.p[k] + call_base;
    for (size_t i = 0; i < kept; i++) out->push_back(WaveRecord{c, sorted[a + i]});
  }
}

// A wave whose host dedup is still to run.  The plain form hands it to the
// next call's run_wave, which runs it after launching its own kernels, so the
// host sort overlaps the device work.  The engine's host read-back buffers
// stay untouched until then: the next wave refills them only after its sync.
// Raw HSPs and scopes a plain call reads back with its totals (40 KB).
constexpr uint32_t kRawPrefix = 2048;
constexpr uint32_t kScopePrefix = 64;

struct DeferredDedup {
  bool pending = false;
  uint32_t nraw = 0, n_scopes = 0, call_base = 0;
  std::vector<WaveRecord> *out = nullptr;
  hz_stats *st = nullptr;
  void finish(hz_engine *e) {
    if (!pending) return;
    pending = false;
    host_dedup(e, nraw, n_scopes, call_base, out, st);
  }
};

// With `defer`, a wave deduped on the host leaves that step in *defer (see
// DeferredDedup) and the records of an earlier deferred wave are emitted once
// this wave's kernels are queued; `call_base` is added to the call index of
// every record the wave emits.
int run_wave(hz_engine *e, const HostCall *hc, size_t n, const uint64_t *seeds, int transitions,
             std::vector<WaveRecord> *out, hz_stats *st, bool device_dedup, bool graph = false,
             DeferredDedup *defer = nullptr, uint32_t call_base = 0) {
  if (n == 0) return HZ_OK;
  cudaStream_t s = e->st;
  uint64_t npos = 0;
  TRY(e->h_calls.ensure(n));
  for (size_t i = 0; i < n; i++) {
    const StagedQuery &q = e->queries[hc[i].query];
    CallDev &c = e->h_calls.p[i];
    c.qoff = hc[i].strand ? q.off_r : q.off_f;
    c.qlen = q.len;
    c.start = hc[i].start;
    c.pos_off = (uint32_t)npos;
    npos += hc[i].end - hc[i].start;
  }
  if (npos == 0) return HZ_OK;
  if (npos >= 0x7FFFFFFFull) return fail(HZ_E_INVALID, "a wave of %llu seed positions exceeds 2^31", (unsigned long long)npos);
  TRY(e->calls.ensure(n, s));
  TRY(e->pos_hits.ensure(npos, s));
  uint64_t tiles = scan_tiles(npos);
  TRY(e->np_partial.ensure(tiles + 1, s));
  TRY(e->np_grand.ensure(1, s));
  TRY(e->np_excl.ensure(npos + 1, s));
  TRY(e->np_pos.ensure(npos + 1, s));
  TRY(e->pos_kmer.ensure(npos, s));
  TRY(e->np_kmer.ensure(npos + 1, s));
  TRY(e->call_hit_lo.ensure(n + 1, s));
  TRY(e->call_nz_lo.ensure(n + 1, s));
  TRY(e->tot.ensure(1, s));
  TRY(e->h_tot.ensure(1));
  CK(cudaMemcpyAsync(e->calls.p, e->h_calls.p, n * sizeof(CallDev), cudaMemcpyHostToDevice, s));

  WaveIn w;
  w.ref = e->ref.base();
  w.rlen = e->rlen;
  w.qbuf = e->qstore.base();
  w.index_table = e->index_table.p;
  w.pos_table = e->pos_table.p;
  w.calls = e->calls.p;
  w.ncalls = (uint32_t)n;
  w.npos = (uint32_t)npos;
  w.seeds = seeds;
  w.shape = e->shape;
  w.per_pos = seeds ? 1u : e->per_pos(transitions);
  w.occ_cap = e->cfg.occ_cap;
  w.nbr_hits = e->has_nbr ? e->nbr_hits.p : nullptr;
  const bool packed_q = e->qry_p.valid && e->shape.size <= 32 && e->qry_p.half >= e->qstore.len;
  w.qp2 = packed_q ? e->qry_p.half_ptr(0) : nullptr;
  w.pos_kmer = e->pos_kmer.p;

  for (int attempt = 0; attempt < 8; attempt++) {  // each rerun fixes every capacity it found short
    uint32_t scope_cap = std::max<uint32_t>(e->scope_cap, (uint32_t)n * 2 + 16);
    TRY(e->scope_lo.ensure(scope_cap + 1, s));
    TRY(e->scope_call.ensure(scope_cap + 1, s));
    TRY(e->cand.ensure(e->cand_cap, s));
    TRY(e->raw.ensure(e->raw_cap, s));
    TRY(e->raw_scope.ensure(e->raw_cap, s));
    TRY(e->tile_first.ensure(e->tile_cap, s));
    TRY(e->tile_call.ensure(e->tile_cap, s));
    // The wave's device chain: no host round trip between its launches, so
    // the batched form can replay it as one CUDA graph.
    auto chain = [&]() -> int {
      CK(cudaMemsetAsync(e->tot.p, 0, sizeof(WaveTotals), s));

      TRY(e->launch("lookup_count", [&] {
        const uint32_t ch = lookup_chunks(npos);
        const uint64_t span = (uint64_t)ch * kCountPerBlock;
        lookup_count_kernel<<<(unsigned)((npos + span - 1) / span), kCountThreads, 0, s>>>(w, ch, e->pos_hits.p,
                                                                                          e->tot.p);
      }));
      TRY(e->launch(
          "np_scan",
          [&] {
            np_reduce_kernel<<<(unsigned)tiles, kScanThreads, 0, s>>>(e->pos_hits.p, npos, e->np_partial.p);
            scan_partials_kernel<HitNz><<<1, kScanThreads, 0, s>>>(e->np_partial.p, tiles, e->np_grand.p);
            np_emit_kernel<<<(unsigned)tiles, kScanThreads, 0, s>>>(e->pos_hits.p, npos, e->np_partial.p,
                                                                    e->np_excl.p, e->np_pos.p, e->pos_kmer.p,
                                                                    e->np_kmer.p);
            np_totals_kernel<<<1, 32, 0, s>>>(e->np_grand.p, e->tot.p, e->np_excl.p);
          },
          4));
      TRY(e->launch("tile_table", [&] {
        tile_table_kernel<<<grid_for(npos, 256, e->sm_count * 8), 256, 0, s>>>(
            e->np_excl.p, e->pos_hits.p, e->np_pos.p, e->calls.p, (uint32_t)n, e->tot.p, (uint32_t)e->gate_tile,
            e->tile_first.p, e->tile_call.p, e->tile_cap);
      }));
      TRY(e->launch("scopes", [&] {
        scopes_kernel<<<1, kScopeThreads, 0, s>>>(w, e->np_excl.p, e->np_pos.p, e->tot.p, e->max_hits,
                                                  e->call_hit_lo.p, e->call_nz_lo.p, e->scope_lo.p, e->scope_call.p,
                                                  scope_cap);
      }));
      GateArgs ga;
      ga.w = w;
      ga.np_excl = e->np_excl.p;
      ga.np_pos = e->np_pos.p;
      ga.np_kmer = e->np_kmer.p;
      ga.scope_lo = e->scope_lo.p;
      ga.scope_cap = scope_cap;
      ga.tot = e->tot.p;
      memcpy(ga.sub, e->cfg.sub_mat, sizeof(ga.sub));
      ga.xdrop = e->cfg.xdrop;
      ga.hspthresh = e->cfg.hspthresh;
      ga.cap = e->gate_cap;
      {
        int32_t top = 0;  // the largest substitution score (0 if none is positive)
        for (int i = 0; i < 64; i++) top = std::max(top, e->cfg.sub_mat[i]);
        ga.late_max_safe = 7ll * top <= (long long)e->cfg.xdrop;
        ga.total_exact = 2ll * (long long)e->gate_cap * top < (1ll << 24);
      }
      ga.cand = e->cand.p;
      ga.cand_cap = e->cand_cap;
      ga.tile_first = e->tile_first.p;
      ga.tile_call = e->tile_call.p;
      if (gate2_usable(e)) {
        switch (e->gate_tile) {
          case 64: TRY(launch_gate2<64>(e, ga)); break;
          case 256: TRY(launch_gate2<256>(e, ga)); break;
          default: TRY(launch_gate2<128>(e, ga)); break;
        }
        TRY(launch_long(e, ga));
      } else {
        switch (e->gate_tile) {
          case 64: TRY(launch_gate<64>(e, ga)); break;
          case 256: TRY(launch_gate<256>(e, ga)); break;
          default: TRY(launch_gate<128>(e, ga)); break;
        }
      }
      ExactArgs xa;
      xa.ref = w.ref;
      xa.rlen = w.rlen;
      xa.qbuf = w.qbuf;
      xa.calls = w.calls;
      xa.cand = e->cand.p;
      xa.cand_cap = e->cand_cap;
      xa.tot = e->tot.p;
      memcpy(xa.sub, e->cfg.sub_mat, sizeof(xa.sub));
      xa.xdrop = e->cfg.xdrop;
      xa.hspthresh = e->cfg.hspthresh;
      xa.noentropy = e->cfg.noentropy ? 1u : 0u;
      xa.raw = e->raw.p;
      xa.raw_scope = e->raw_scope.p;
      xa.raw_cap = e->raw_cap;
      TRY(e->launch("exact", [&] {
        exact_kernel<<<(unsigned)(e->sm_count * 8), kExactThreads, 0, s>>>(xa);
      }));
      CK(cudaMemcpyAsync(e->h_tot.p, e->tot.p, sizeof(WaveTotals), cudaMemcpyDeviceToHost, s));
      return HZ_OK;
    };
    if (graph) TRY(run_captured(e, chain));
    else TRY(chain());
    if (defer) defer->finish(e);  // the previous call's host dedup, while this call's kernels run
    // A single-call wave (the plain form) reads back the first raw HSPs and
    // scopes with its totals, so one with few raw HSPs (the usual case) needs
    // one sync, not two.
    uint32_t pre_raw = 0, pre_scopes = 0;
    if (n == 1 && !device_dedup) {
      pre_raw = std::min<uint32_t>(kRawPrefix, e->raw_cap);
      pre_scopes = std::min<uint32_t>(kScopePrefix, scope_cap + 1);
      TRY(e->h_raw.ensure(pre_raw));
      TRY(e->h_raw_scope.ensure(pre_raw));
      TRY(e->h_scope_call.ensure(pre_scopes));
      CK(cudaMemcpyAsync(e->h_raw.p, e->raw.p, (size_t)pre_raw * sizeof(SegmentPair), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(e->h_raw_scope.p, e->raw_scope.p, (size_t)pre_raw * 4, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(e->h_scope_call.p, e->scope_call.p, (size_t)pre_scopes * 4, cudaMemcpyDeviceToHost, s));
    }
    TRY(e->sync());
    WaveTotals t = *e->h_tot.p;
    if (t.status & 2u) return fail(HZ_E_INVALID, "a call holds 2^32 or more seed hits; num_hits is a u32 in the reference");
    if (t.status & 1u)
      return fail(HZ_E_INVALID, "the first seed of a call holds more than max_hits=%u hits; the reference's MAX_HITS "
                                "walk has no valid cut there", e->max_hits);
    bool again = false;
    // a wave of several calls holding more hits than wave_hits_cap is cut
    // smaller (run_calls halves its position budget), so the grow-only wave
    // buffers stay bounded on repeat-dense input
    if (n > 1 && t.hits > e->wave_hits_cap) return kSplitWave;
    if (t.status & 4u) {  // the gate skipped the wave: its tile table was too small
      e->tile_cap = (uint32_t)std::min<uint64_t>(t.hits / (uint64_t)e->gate_tile + 1024, 0xFFFFFFF0ull);
      again = true;
    }
    if (t.n_scopes > scope_cap) {
      e->scope_cap = t.n_scopes + 16;
      again = true;
    }
    if (t.cand > e->cand_cap) {
      e->cand_cap = t.cand + t.cand / 4 + 1024;
      again = true;
    }
    if (t.raw > e->raw_cap) {
      e->raw_cap = t.raw + t.raw / 4 + 1024;
      again = true;
    }
    if (again) continue;  // a capacity was too small: run the wave again with larger buffers

    // per-scope dedup on the host, in scope order
    uint32_t nraw = t.raw;
    e->cand_seen += t.cand;
    if (st) {
      st->hits += t.hits;
      st->cells += t.cells;
      st->seeds += t.valid * w.per_pos;
      st->raw_hsps += nraw;
      st->calls += n;
    }
    if (nraw == 0) return HZ_OK;
    // per-call waves (the plain form) dedup on the host like the reference,
    // unless the call holds so many raw HSPs that the device sort is faster
    if (device_dedup || (e->device_dedup && nraw >= e->device_dedup_min))
      return dedup_on_device(e, nraw, t.n_scopes, call_base, out, st);
    if (nraw > pre_raw || t.n_scopes > pre_scopes) {  // not all read back with the totals
      TRY(e->h_raw.ensure(nraw));
      TRY(e->h_raw_scope.ensure(nraw));
      TRY(e->h_scope_call.ensure(t.n_scopes + 1));
      CK(cudaMemcpyAsync(e->h_raw.p, e->raw.p, (size_t)nraw * sizeof(SegmentPair), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(e->h_raw_scope.p, e->raw_scope.p, (size_t)nraw * 4, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(e->h_scope_call.p, e->scope_call.p, (size_t)t.n_scopes * 4, cudaMemcpyDeviceToHost, s));
      TRY(e->sync());
    }
    if (defer) {
      defer->pending = true;
      defer->nraw = nraw;
      defer->n_scopes = t.n_scopes;
      defer->call_base = call_base;
      defer->out = out;
      defer->st = st;
      return HZ_OK;
    }
    host_dedup(e, nraw, t.n_scopes, call_base, out, st);
    return HZ_OK;
  }
  return fail(HZ_E_OOM, "wave buffers kept overflowing");
}

// The calls of one staged query in the reference's batch order: per LASTZ
// interval (src/sequence.rs:322-334), the plus WGA chunks then the minus
// chunks over (qbl - end, qbl - start) (src/run.rs:278-299, chunks
// src/seed.rs:488-496).
void query_calls(const hz_engine *e, uint32_t qid, std::vector<HostCall> *out) {
  uint64_t qlen = e->queries[qid].len;
  uint32_t ss = e->shape.size;
  if (qlen <= ss) return;
  uint32_t end_pos = (uint32_t)(qlen - ss), qbl = end_pos;
  uint32_t iv = 0;
  for (uint64_t cur = 0; cur < end_pos; cur += e->cfg.interval, iv++) {
    uint32_t is = (uint32_t)cur, ie = (uint32_t)std::min<uint64_t>(end_pos, cur + e->cfg.interval);
    for (uint32_t rev = 0; rev < 2; rev++) {
      if (!(e->cfg.strand & (1u << rev))) continue;
      uint32_t a = rev ? qbl - ie : is, b = rev ? qbl - is : ie;
      for (uint64_t c = a; c < b; c += e->cfg.wga_chunk)
        out->push_back(HostCall{qid, iv, rev, (uint32_t)c, (uint32_t)std::min<uint64_t>(c + e->cfg.wga_chunk, (uint64_t)b + 1)});
    }
  }
}

// The per-k-mer neighbourhood hit counts, for seed patterns of at most 14
// care positions (a 4^k table of at most 1 GB); larger patterns look up
// every seed of a position instead.
int build_nbr_hits(hz_engine *e, uint64_t index_len) {
  e->has_nbr = false;
  if (e->shape.kmer_size > 14) return HZ_OK;
  cudaStream_t s = e->st;
  TRY(e->nbr_hits.ensure(index_len, s));
  const uint32_t *idx = e->index_table.p;
  uint32_t *out = e->nbr_hits.p;
  const uint32_t ks = e->shape.kmer_size, cap = e->cfg.occ_cap;
  TRY(e->launch("nbr_hits", [&] {
    nbr_hits_kernel<<<grid_for(index_len, 256), 256, 0, s>>>(idx, index_len, ks, cap, out);
  }));
  e->has_nbr = true;
  return HZ_OK;
}

// Replaces the query store with `nq` ASCII blocks; each is encoded forward
// and reverse-complemented on the device.
int stage_ascii(hz_engine *e, const uint8_t *const *ascii, const uint64_t *lens, uint32_t nq) {
  uint64_t total = 0;
  std::vector<StagedQuery> qs(nq);
  for (uint32_t i = 0; i < nq; i++) {
    if (lens[i] > 0xFFFFFFFFull) return fail(HZ_E_INVALID, "query block %u exceeds u32 coordinates", i);
    // every strand starts 16-byte aligned, with at least kPad bytes after it
    qs[i].len = (uint32_t)lens[i];
    qs[i].off_f = (uint32_t)total;
    total = (total + lens[i] + kPad + 15) & ~15ull;
    qs[i].off_r = (uint32_t)total;
    total = (total + lens[i] + kPad + 15) & ~15ull;
  }
  if (total >= 0xFFFFFFFFull) return fail(HZ_E_INVALID, "staged queries exceed 4 GB");
  cudaStream_t s = e->st;
  TRY(e->qstore.ensure(total, s));
  uint64_t maxlen = 0;
  for (uint32_t i = 0; i < nq; i++) maxlen = std::max<uint64_t>(maxlen, lens[i]);
  TRY(e->qascii.ensure(maxlen + 16, s));
  CK(cudaMemsetAsync(e->qstore.base(), 0, total, s));
  for (uint32_t i = 0; i < nq; i++) {
    if (!lens[i]) continue;
    CK(cudaMemcpyAsync(e->qascii.p, ascii[i], lens[i], cudaMemcpyHostToDevice, s));
    uint8_t *f = e->qstore.base() + qs[i].off_f, *r = e->qstore.base() + qs[i].off_r;
    uint64_t len = lens[i];
    TRY(e->launch("encode", [&] {
      encode_kernel<<<grid_for(len / 4 + 1, 256), 256, 0, s>>>(e->qascii.p, len, f, r);
    }));
  }
  TRY(pack_seq(e, e->qstore.base(), total, &e->qry_p));
  TRY(e->sync());
  e->queries = qs;
  e->cur_query = 0;
  e->has_query = nq > 0;
  e->slot[0].kind = e->slot[1].kind = 0;
  return HZ_OK;
}

// The batched form over every staged query: the calls, query-major, cut into
// waves of at most wave_positions seed positions at call boundaries.
// *recs[k].call indexes *calls.
// Runs `calls` through batched waves of at most wave_positions positions.
int run_calls(hz_engine *e, std::vector<HostCall> *calls, std::vector<WaveRecord> *recs, hz_stats *st) {
  size_t i = 0;
  uint64_t budget = e->wave_positions;  // halved whenever a wave holds more than wave_hits_cap hits
  while (i < calls->size()) {
    size_t j = i;
    uint64_t npos = 0;
    while (j < calls->size() && (j == i || npos + ((*calls)[j].end - (*calls)[j].start) <= budget)) {
      npos += (*calls)[j].end - (*calls)[j].start;
      j++;
    }
    size_t before = recs->size();
    const int rc = run_wave(e, calls->data() + i, j - i, nullptr, e->cfg.transitions, recs, st, e->device_dedup,
                            e->use_graph);
    if (rc == kSplitWave) {  // nothing of the wave was kept: run its calls in smaller waves
      budget = std::max<uint64_t>(budget / 2, 1);
      continue;
    }
    TRY(rc);
    for (size_t k = before; k < recs->size(); k++) (*recs)[k].call += (uint32_t)i;
    i = j;
  }
  return HZ_OK;
}

int run_all_staged(hz_engine *e, std::vector<HostCall> *calls, std::vector<WaveRecord> *recs, hz_stats *st) {
  for (uint32_t q = 0; q < e->queries.size(); q++) query_calls(e, q, calls);
  return run_calls(e, calls, recs, st);
}

int check_range(hz_engine *e, uint32_t start, uint32_t end) {
  if (end < start) return fail(HZ_E_INVALID, "seed range [%u, %u) is reversed", start, end);
  uint32_t qlen = e->queries.empty() ? 0 : e->queries[e->cur_query].len;
  if (end > start && (uint64_t)end + e->shape.size - 1 > qlen)
    return fail(HZ_E_INVALID, "seed range [%u, %u) exceeds query length %u", start, end, qlen);
  return HZ_OK;
}

// f(begin, end) over [0, n) on up to 16 host threads (one for small n, or
// if a thread cannot be started): output copies of hundreds of millions of
// records are bound by first-touch page faults, which threads take in
// parallel.
template <typename F> void parallel_ranges(size_t n, F f) {
  const size_t kMinPerThread = 1u << 20;
  unsigned t = std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 16u);
  t = (unsigned)std::min<size_t>(t, n / kMinPerThread);
  if (t <= 1) {
    f((size_t)0, n);
    return;
  }
  const size_t per = (n + t - 1) / t;
  std::vector<std::thread> th;
  size_t done = 0;  // ranges below `done` have a thread
  try {
    for (unsigned i = 0; i < t; i++) {
      const size_t a = i * per, b = std::min(n, a + per);
      if (a >= b) break;
      th.emplace_back(f, a, b);
      done = b;
    }
  } catch (...) {
  }
  if (done < n) f(done, n);
  for (auto &x : th) x.join();
}

int copy_out_segments(const std::vector<WaveRecord> &recs, hz_segment_pair **out, uint64_t *n) {
  *out = nullptr;
  *n = recs.size();
  if (recs.empty()) return HZ_OK;
  *out = (hz_segment_pair *)malloc(recs.size() * sizeof(hz_segment_pair));
  if (!*out) return fail(HZ_E_OOM, "host allocation");
  hz_segment_pair *o = *out;
  parallel_ranges(recs.size(), [&](size_t a, size_t b) {
    for (size_t i = a; i < b; i++) o[i] = recs[i].h;
  });
  return HZ_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

const char *hz_last_error(void) { return g_err.c_str(); }

void hz_free(void *p) { free(p); }

int hz_shape_info(const char *seed, uint32_t *size, uint32_t *kmer_size) {
  ShapeDev sh;
  if (!seed) return fail(HZ_E_INVALID, "null seed");
  TRY(parse_shape(seed, &sh));
  if (size) *size = sh.size;
  if (kmer_size) *kmer_size = sh.kmer_size;
  return HZ_OK;
}

int hz_engine_create(const hz_config *cfg, int device, hz_engine **out) {
  if (!cfg || !out) return fail(HZ_E_INVALID, "null argument");
  *out = nullptr;
  ShapeDev sh;
  char seed[65];
  memcpy(seed, cfg->seed, 64);
  seed[64] = 0;
  TRY(parse_shape(seed[0] ? seed : "12of19", &sh));
  if (cfg->strand == 0 || cfg->strand > 3) return fail(HZ_E_INVALID, "strand must be 1 (plus), 2 (minus) or 3 (both)");
  int ndev = 0;
  cudaError_t err = cudaGetDeviceCount(&ndev);
  if (err != cudaSuccess || ndev == 0)
    return fail(HZ_E_CUDA, "no CUDA device available (%s); this library has no CPU path",
                err != cudaSuccess ? cudaGetErrorString(err) : "0 devices");
  if (device < 0 || device >= ndev) return fail(HZ_E_INVALID, "device %d out of range (%d devices)", device, ndev);
  CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(HZ_E_CUDA, "device %d is sm_%d%d; this build targets sm_100a (B200)", device, prop.major, prop.minor);
  hz_engine *e = new hz_engine();
  e->device = device;
  e->sm_count = prop.multiProcessorCount;
  e->cfg = *cfg;
  e->cfg.seed[63] = 0;
  e->shape = sh;
  if (e->cfg.step == 0) e->cfg.step = 1;
  if (e->cfg.wga_chunk == 0) e->cfg.wga_chunk = 250000;
  if (e->cfg.interval == 0) e->cfg.interval = 10000000;
  if (cfg->max_hits > 0) {
    e->max_hits = cfg->max_hits;
  } else {
    // default_max_hits (src/gpu/mod.rs:2422-2433): 4194304 x total GiB, in f32
    float gib = (float)prop.totalGlobalMem / 1073741824.0f;
    double v = (double)(4194304.0f * gib);
    uint64_t m = (uint64_t)v;
    e->max_hits = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(m, 1), 0xFFFFFFFFull);
  }
  cudaError_t se = cudaStreamCreateWithFlags(&e->own_st, cudaStreamNonBlocking);
  if (se != cudaSuccess) {
    delete e;
    return fail(HZ_E_CUDA, "stream: %s", cudaGetErrorString(se));
  }
  e->st = e->own_st;
  uint8_t t_enc[256], t_rc[256];
  for (int c = 0; c < 256; c++) {
    t_enc[c] = enc_of((uint8_t)c);
    t_rc[c] = enc_of(c < 128 ? (uint8_t)kRevComp[c] : (uint8_t)'N');
  }
  int rc = HZ_OK;
  if (cudaMemcpyToSymbol(c_enc, t_enc, 256) != cudaSuccess || cudaMemcpyToSymbol(c_enc_rc, t_rc, 256) != cudaSuccess)
    rc = fail(HZ_E_CUDA, "constant tables: %s", cudaGetErrorString(cudaGetLastError()));
  if (rc == HZ_OK) rc = e->ref.ensure(0, e->st);
  if (rc == HZ_OK) rc = e->qstore.ensure(0, e->st);
  if (rc != HZ_OK) {
    hz_engine_destroy(e);
    return rc;
  }
  *out = e;
  return HZ_OK;
}

void hz_engine_destroy(hz_engine *e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->st) cudaStreamSynchronize(e->st);
  if (e->server) hz_serve_stop(e);
  for (hz_engine *w : e->twins) hz_engine_destroy(w);
  e->twins.clear();
  if (e->owns_target) {
    e->ref.buf.release();
    e->index_table.release();
    e->pos_table.release();
    e->nbr_hits.release();
    e->ref_p.release();
  }
  if (!e->aliases_query) {
    e->qstore.buf.release();
    e->qry_p.release();
  }
  e->qascii.release();
  e->build.release();
  for (auto &s : e->slot) s.seeds.release();
  e->calls.release();
  e->pos_hits.release();
  e->np_pos.release();
  e->pos_kmer.release();
  e->np_kmer.release();
  e->call_nz_lo.release();
  e->scope_call.release();
  e->raw_scope.release();
  e->np_excl.release();
  e->call_hit_lo.release();
  e->scope_lo.release();
  e->np_partial.release();
  e->np_grand.release();
  e->tot.release();
  e->cand.release();
  e->raw.release();
  e->h_calls.release();
  e->h_tot.release();
  e->h_raw.release();
  e->h_raw_scope.release();
  e->h_scope_call.release();
  for (auto *b : {&e->d_perm_a, &e->d_perm_b, &e->d_keys_a, &e->d_keys_b, &e->d_keep, &e->d_keep_excl, &e->d_hist,
                  &e->d_hpart, &e->d_total, &e->tile_first, &e->tile_call})
    b->release();
  e->d_out.release();
  e->h_out.release();
  for (auto &pe : e->pending)
    if (pe.pooled) {
      cudaEventDestroy(pe.a);
      cudaEventDestroy(pe.b);
    }
  for (auto ev : e->event_pool) cudaEventDestroy(ev);
  for (auto &ge : e->graph_events) {
    cudaEventDestroy(ge.second.first);
    cudaEventDestroy(ge.second.second);
  }
  if (e->wave_exec) cudaGraphExecDestroy(e->wave_exec);
  if (e->own_st) cudaStreamDestroy(e->own_st);
  delete e;
}

int hz_engine_load_tables(hz_engine *e, const uint32_t *index_table, uint64_t index_len, const uint32_t *pos_table,
                          uint64_t pos_len, const uint8_t *ref_seq, uint64_t ref_len) {
  if (!e || !index_table || (ref_len && !ref_seq) || (pos_len && !pos_table)) return fail(HZ_E_INVALID, "null argument");
  if (e->server) return fail(HZ_E_STATE, "the serving loop is running on this target");
  if (index_len != (1ull << (2 * e->shape.kmer_size)))
    return fail(HZ_E_INVALID, "index_table has %llu entries, the seed needs 4^%u", (unsigned long long)index_len,
                e->shape.kmer_size);
  if (ref_len > 0xFFFFFFFFull) return fail(HZ_E_INVALID, "reference block exceeds u32 coordinates");
  if (index_table[index_len - 1] != pos_len)
    return fail(HZ_E_INVALID, "index_table total %u != pos_table length %llu", index_table[index_len - 1],
                (unsigned long long)pos_len);
  // The kernels trust these invariants for their address arithmetic, so a
  // malformed table is refused here rather than read out of bounds.
  for (uint64_t k = 1; k < index_len; k++)
    if (index_table[k] < index_table[k - 1])
      return fail(HZ_E_INVALID, "index_table decreases at bucket %llu", (unsigned long long)k);
  for (uint64_t i = 0; i < pos_len; i++)
    if ((uint64_t)pos_table[i] + e->shape.size > ref_len)
      return fail(HZ_E_INVALID, "pos_table[%llu]=%u leaves no full seed window in a %llu-base reference",
                  (unsigned long long)i, pos_table[i], (unsigned long long)ref_len);
  for (uint64_t i = 0; i < ref_len; i++)
    if (ref_seq[i] > 7) return fail(HZ_E_INVALID, "ref_seq[%llu]=%u is not a device-alphabet code", (unsigned long long)i, ref_seq[i]);
  TRY(set_device(e));
  cudaStream_t s = e->st;
  TRY(e->index_table.ensure(index_len, s));
  TRY(e->pos_table.ensure(pos_len + 1, s));
  TRY(e->ref.ensure(ref_len, s));
  CK(cudaMemcpyAsync(e->index_table.p, index_table, index_len * 4, cudaMemcpyHostToDevice, s));
  if (pos_len) CK(cudaMemcpyAsync(e->pos_table.p, pos_table, pos_len * 4, cudaMemcpyHostToDevice, s));
  if (ref_len) CK(cudaMemcpyAsync(e->ref.base(), ref_seq, ref_len, cudaMemcpyHostToDevice, s));
  TRY(pack_seq(e, e->ref.base(), ref_len, &e->ref_p));
  TRY(e->sync());
  TRY(build_nbr_hits(e, index_len));
  e->index_len = index_len;
  e->n_pos = pos_len;
  e->rlen = (uint32_t)ref_len;
  e->has_target = true;
  return HZ_OK;
}

int hz_engine_load_target(hz_engine *e, const uint8_t *ref_ascii, uint64_t len) {
  if (!e || (!ref_ascii && len)) return fail(HZ_E_INVALID, "null argument");
  if (e->server) return fail(HZ_E_STATE, "the serving loop is running on this target");
  if (len > 0xFFFFFFFFull) return fail(HZ_E_INVALID, "reference block exceeds u32 coordinates");
  TRY(set_device(e));
  cudaStream_t st = e->st;
  const ShapeDev &sh = e->shape;
  uint64_t index_len = 1ull << (2 * sh.kmer_size);
  uint32_t step = e->cfg.step;
  uint64_t offset = (sh.size + 1) % step;
  uint64_t start_offset = step - offset;
  uint64_t num_steps = (len + offset) > sh.size ? (len + offset - sh.size) / step : 0;

  // ASCII -> device codes
  auto &bs = e->build;
  DBuf<uint8_t> &ascii = bs.ascii, &junk = bs.junk;
  TRY(ascii.ensure(len + 1, st));
  TRY(e->ref.ensure(len, st));
  TRY(junk.ensure(len + 1, st));
  if (len) CK(cudaMemcpyAsync(ascii.p, ref_ascii, len, cudaMemcpyHostToDevice, st));
  uint8_t *codes = e->ref.base();
  if (len)
    TRY(e->launch("encode", [&] {
      encode_kernel<<<grid_for(len / 4 + 1, 256), 256, 0, st>>>(ascii.p, len, codes, junk.p);
    }));
  TRY(e->index_table.ensure(index_len, st));
  CK(cudaMemsetAsync(e->index_table.p, 0, index_len * 4, st));

  DBuf<uint32_t> &kmers = bs.kmers, &flags = bs.flags, &keys = bs.keys, &vals = bs.vals, &keys2 = bs.keys2,
                 &vals2 = bs.vals2, &partial = bs.partial, &total = bs.total, &hist = bs.hist,
                 &hpartial = bs.hpartial;
  uint64_t n_valid = 0;
  if (num_steps) {
    TRY(kmers.ensure(num_steps, st));
    TRY(flags.ensure(num_steps, st));
    TRY(partial.ensure(scan_tiles(num_steps) + 1, st));
    TRY(total.ensure(1, st));
    TRY(e->launch("ref_kmer", [&] {
      ref_kmer_kernel<<<grid_for(num_steps, 256), 256, 0, st>>>(codes, num_steps, start_offset, step, sh, kmers.p,
                                                                flags.p);
    }));
    TRY(e->launch("ref_scan", [&] { exclusive_scan<uint32_t>(flags.p, flags.p, num_steps, partial.p, total.p, st); }, 3));
    uint32_t tot = 0;
    CK(cudaMemcpyAsync(&tot, total.p, 4, cudaMemcpyDeviceToHost, st));
    TRY(e->sync());
    n_valid = tot;
    TRY(keys.ensure(n_valid + 1, st));
    TRY(vals.ensure(n_valid + 1, st));
    TRY(e->launch("ref_compact", [&] {
      ref_compact_kernel<<<grid_for(num_steps, 256), 256, 0, st>>>(kmers.p, flags.p, num_steps, start_offset, step,
                                                                   keys.p, vals.p, e->index_table.p);
    }));
    // stable radix sort by k-mer, 8 bits per pass: each bucket keeps
    // ascending position order (src/seed.rs:157-170)
    if (n_valid) {
      TRY(keys2.ensure(n_valid + 1, st));
      TRY(vals2.ensure(n_valid + 1, st));
      uint64_t rtiles = (n_valid + kRadixTile - 1) / kRadixTile;
      TRY(hist.ensure(rtiles * kRadixBins, st));
      TRY(hpartial.ensure(scan_tiles(rtiles * kRadixBins) + 1, st));
      int bits = 2 * (int)sh.kmer_size;
      uint32_t *ka = keys.p, *va = vals.p, *kb = keys2.p, *vb = vals2.p;
      for (int shift = 0; shift < bits; shift += 8) {
        TRY(e->launch("radix_hist", [&] {
          radix_hist_kernel<<<(unsigned)rtiles, kRadixThreads, 0, st>>>(ka, n_valid, shift, hist.p, rtiles);
        }));
        TRY(e->launch("radix_scan", [&] {
          exclusive_scan<uint32_t>(hist.p, hist.p, rtiles * kRadixBins, hpartial.p, total.p, st);
        }, 3));
        TRY(e->launch("radix_scatter", [&] {
          radix_scatter_kernel<<<(unsigned)rtiles, kRadixThreads, 0, st>>>(ka, va, n_valid, shift, hist.p, rtiles, kb,
                                                                          vb);
        }));
        std::swap(ka, kb);
        std::swap(va, vb);
      }
      TRY(e->pos_table.ensure(n_valid + 1, st));
      CK(cudaMemcpyAsync(e->pos_table.p, va, n_valid * 4, cudaMemcpyDeviceToDevice, st));
    }
  }
  TRY(e->pos_table.ensure(1, st));
  // index_table = inclusive cumulative bucket counts (src/seed.rs:162-164)
  {
    DBuf<uint32_t> &excl = bs.excl, &ipart = bs.ipart;
    TRY(excl.ensure(index_len, st));
    TRY(ipart.ensure(scan_tiles(index_len) + 1, st));
    TRY(total.ensure(1, st));
    TRY(e->launch("index_scan", [&] {
      exclusive_scan<uint32_t>(e->index_table.p, excl.p, index_len, ipart.p, total.p, st);
    }, 3));
    TRY(e->launch("index_add", [&] {
      add_counts_kernel<<<grid_for(index_len, 256), 256, 0, st>>>(excl.p, e->index_table.p, index_len);
    }));
    CK(cudaMemcpyAsync(e->index_table.p, excl.p, index_len * 4, cudaMemcpyDeviceToDevice, st));
    TRY(e->sync());
  }
  if (bs.bytes() > kKeepBuildScratch) bs.release();
  TRY(pack_seq(e, e->ref.base(), len, &e->ref_p));
  TRY(build_nbr_hits(e, index_len));
  e->index_len = index_len;
  e->n_pos = n_valid;
  e->rlen = (uint32_t)len;
  e->has_target = true;
  return HZ_OK;
}

int hz_engine_read_tables(hz_engine *e, uint32_t *index_table, uint64_t *index_len, uint32_t *pos_table,
                          uint64_t *pos_len) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  if (!e->has_target) return fail(HZ_E_STATE, "no target loaded");
  TRY(set_device(e));
  if (index_len) *index_len = e->index_len;
  if (pos_len) *pos_len = e->n_pos;
  if (index_table) CK(cudaMemcpyAsync(index_table, e->index_table.p, e->index_len * 4, cudaMemcpyDeviceToHost, e->st));
  if (pos_table && e->n_pos) CK(cudaMemcpyAsync(pos_table, e->pos_table.p, e->n_pos * 4, cudaMemcpyDeviceToHost, e->st));
  return e->sync();
}

int hz_swap_query(hz_engine *e, const uint8_t *query, const uint8_t *query_rc, uint64_t len) {
  if (!e || (len && (!query || !query_rc))) return fail(HZ_E_INVALID, "null argument");
  if (len > 0xFFFFFFFFull) return fail(HZ_E_INVALID, "query block exceeds u32 coordinates");
  for (uint64_t i = 0; i < len; i++)
    if (query[i] > 7 || query_rc[i] > 7) return fail(HZ_E_INVALID, "query byte %llu is not a device-alphabet code", (unsigned long long)i);
  TRY(set_device(e));
  StagedQuery q;
  q.len = (uint32_t)len;
  q.off_f = 0;
  q.off_r = (uint32_t)((len + kPad + 15) & ~15ull);
  uint64_t total = q.off_r + len + kPad;
  TRY(e->qstore.ensure(total, e->st));
  CK(cudaMemsetAsync(e->qstore.base(), 0, total, e->st));
  if (len) {
    CK(cudaMemcpyAsync(e->qstore.base() + q.off_f, query, len, cudaMemcpyHostToDevice, e->st));
    CK(cudaMemcpyAsync(e->qstore.base() + q.off_r, query_rc, len, cudaMemcpyHostToDevice, e->st));
  }
  TRY(pack_seq(e, e->qstore.base(), total, &e->qry_p));
  TRY(e->sync());
  e->queries.assign(1, q);
  e->cur_query = 0;
  e->has_query = true;
  e->slot[0].kind = e->slot[1].kind = 0;
  return HZ_OK;
}

int hz_swap_query_ascii(hz_engine *e, const uint8_t *q, uint64_t len) {
  if (!e || (len && !q)) return fail(HZ_E_INVALID, "null argument");
  TRY(set_device(e));
  return stage_ascii(e, &q, &len, 1);
}

int hz_upload_seeds(hz_engine *e, uint32_t slot, const uint64_t *seeds, uint64_t n) {
  if (!e || slot > 1 || (n && !seeds)) return fail(HZ_E_INVALID, "bad argument");
  if (!e->has_query) return fail(HZ_E_STATE, "Engine has no query: swap_query() must be called before upload_seeds()");
  if (n >= 0x7FFFFFFFull) return fail(HZ_E_INVALID, "too many seeds in one call");
  uint32_t qlen = e->queries[e->cur_query].len;
  uint32_t max_pos = qlen >= e->shape.size ? qlen - e->shape.size : 0;
  for (uint64_t i = 0; i < n; i++) {
    uint64_t k = seeds[i] >> 32;
    if (k >= e->index_len || (uint32_t)seeds[i] > max_pos || qlen < e->shape.size)
      return fail(HZ_E_INVALID, "seed %llu (k-mer %llu, position %u) lies outside the seed table or the query",
                  (unsigned long long)i, (unsigned long long)k, (uint32_t)seeds[i]);
  }
  TRY(set_device(e));
  Slot &s = e->slot[slot];
  TRY(s.seeds.ensure(n + 1, e->st));
  if (n) CK(cudaMemcpyAsync(s.seeds.p, seeds, n * 8, cudaMemcpyHostToDevice, e->st));
  TRY(e->sync());
  s.kind = 1;
  s.n = n;
  return HZ_OK;
}

// Counts the valid windows of [start, end) so the seed count is known as
// chunk_seeds would report it; the lookup itself runs in seed_and_filter.
int hz_generate_seeds(hz_engine *e, uint32_t slot, int rev, uint32_t start, uint32_t end, int transitions,
                      uint64_t *n_seeds) {
  if (!e || slot > 1) return fail(HZ_E_INVALID, "bad argument");
  if (!e->has_query) return fail(HZ_E_STATE, "Engine has no query: swap_query() must be called before generate_seeds()");
  if (!e->has_target) return fail(HZ_E_STATE, "no target loaded");
  TRY(check_range(e, start, end));
  TRY(set_device(e));
  Slot &s = e->slot[slot];
  s.kind = 2;
  s.rev = rev ? 1 : 0;
  s.start = start;
  s.end = end;
  s.transitions = transitions ? 1 : 0;
  uint64_t nv = 0;
  if (end > start) {
    // the lookup kernel counts valid windows as it goes: run it alone
    const StagedQuery &q = e->queries[e->cur_query];
    TRY(e->h_calls.ensure(1));
    e->h_calls.p[0] = CallDev{s.rev ? q.off_r : q.off_f, q.len, start, 0};
    TRY(e->calls.ensure(1, e->st));
    TRY(e->pos_hits.ensure(end - start, e->st));
    TRY(e->tot.ensure(1, e->st));
    TRY(e->h_tot.ensure(1));
    CK(cudaMemcpyAsync(e->calls.p, e->h_calls.p, sizeof(CallDev), cudaMemcpyHostToDevice, e->st));
    CK(cudaMemsetAsync(e->tot.p, 0, sizeof(WaveTotals), e->st));
    WaveIn w;
    memset(&w, 0, sizeof w);
    w.ref = e->ref.base();
    w.rlen = e->rlen;
    w.qbuf = e->qstore.base();
    w.index_table = e->index_table.p;
    w.pos_table = e->pos_table.p;
    w.calls = e->calls.p;
    w.ncalls = 1;
    w.npos = end - start;
    w.shape = e->shape;
    w.per_pos = e->per_pos(transitions);
    w.occ_cap = e->cfg.occ_cap;
  w.nbr_hits = e->has_nbr ? e->nbr_hits.p : nullptr;
    TRY(e->launch("lookup_count", [&] {
      const uint32_t ch = lookup_chunks(w.npos);
      const uint64_t span = (uint64_t)ch * kCountPerBlock;
      lookup_count_kernel<<<(unsigned)((w.npos + span - 1) / span), kCountThreads, 0, e->st>>>(w, ch, e->pos_hits.p,
                                                                                              e->tot.p);
    }));
    CK(cudaMemcpyAsync(e->h_tot.p, e->tot.p, sizeof(WaveTotals), cudaMemcpyDeviceToHost, e->st));
    TRY(e->sync());
    nv = e->h_tot.p->valid;
  }
  s.n = nv * e->per_pos(transitions);
  if (n_seeds) *n_seeds = s.n;
  return HZ_OK;
}

int hz_seed_and_filter(hz_engine *e, uint32_t slot, int rev, hz_segment_pair **out, uint64_t *n, hz_stats *stats) {
  if (!e || slot > 1 || !out || !n) return fail(HZ_E_INVALID, "bad argument");
  *out = nullptr;
  *n = 0;
  if (!e->has_query)
    return fail(HZ_E_STATE, "Engine has no query: swap_query() must be called before seed_and_filter()");
  if (!e->has_target) return fail(HZ_E_STATE, "no target loaded");
  TRY(set_device(e));
  Slot &s = e->slot[slot];
  if (s.kind == 0) return fail(HZ_E_STATE, "seed slot %u holds no seeds", slot);
  if (s.kind == 2 && s.rev != (rev ? 1 : 0)) return fail(HZ_E_INVALID, "slot %u was generated for the other strand", slot);
  hz_stats local;
  memset(&local, 0, sizeof local);
  std::vector<WaveRecord> recs;
  if (s.kind == 2) {
    HostCall hc{e->cur_query, 0, (uint32_t)(rev ? 1 : 0), s.start, s.end};
    TRY(run_wave(e, &hc, s.end > s.start ? 1 : 0, nullptr, s.transitions, &recs, &local, false));
  } else if (s.n) {
    HostCall hc{e->cur_query, 0, (uint32_t)(rev ? 1 : 0), 0, (uint32_t)s.n};
    TRY(run_wave(e, &hc, 1, s.seeds.p, 0, &recs, &local, false));
  }
  local.seeds = s.n;
  TRY(copy_out_segments(recs, out, n));
  if (stats) *stats = local;
  return HZ_OK;
}

namespace {
void share_target(hz_engine *w, const hz_engine *e);
int clone_shared(hz_engine *e, hz_engine **out);

void add_stats(hz_stats *a, const hz_stats &b) {
  a->seeds += b.seeds;
  a->hits += b.hits;
  a->raw_hsps += b.raw_hsps;
  a->hsps += b.hsps;
  a->cells += b.cells;
  a->calls += b.calls;
}

// The plain pass over `k` workspaces: this engine and k - 1 more (each with
// its own stream and wave buffers over the same target tables and query
// store), each driven by its own host thread and taking the next call from a
// shared counter.  While one waits for its call's read-back and dedups it on
// the host, the others' kernels run, so the device is not idle between calls.
// Calls are independent, so each call's records are the same as on one
// workspace; they are put back in call order.
int run_pass_multi(hz_engine *e, int k, const std::vector<HostCall> &calls, std::vector<WaveRecord> *recs,
                   hz_stats *st) {
  while ((int)e->twins.size() < k - 1) {
    hz_engine *w = nullptr;
    TRY(clone_shared(e, &w));
    w->qstore.buf.release();  // it uses this engine's query store instead
    w->aliases_query = true;
    e->twins.push_back(w);
  }
  std::vector<hz_engine *> ws{e};
  for (int j = 0; j < k - 1; j++) {
    hz_engine *w = e->twins[j];
    share_target(w, e);  // the target, configuration and knobs may have changed since the last pass
    w->qstore.buf.p = e->qstore.buf.p;
    w->qstore.buf.cap = e->qstore.buf.cap;
    w->qstore.len = e->qstore.len;
    w->qry_p = e->qry_p;
    w->queries = e->queries;
    w->cur_query = e->cur_query;
    w->has_query = e->has_query;
    w->profiling = e->profiling;
    ws.push_back(w);
  }
  std::vector<uint64_t> launches0(ws.size());
  for (size_t j = 0; j < ws.size(); j++) launches0[j] = ws[j]->launches;

  std::vector<std::vector<WaveRecord>> per(calls.size());
  std::atomic<size_t> next{0};
  std::atomic<bool> stop{false};
  // calls an extra workspace could not finish for lack of device memory;
  // this engine runs them once the others are done
  std::vector<size_t> orphans;
  std::mutex orphans_mu;
  auto drive = [&](hz_engine *x, hz_stats *sx, bool extra) -> int {
    for (;;) {
      if (stop.load()) return HZ_OK;
      size_t i = next.fetch_add(1);
      if (i >= calls.size()) return HZ_OK;
      hz_stats one;  // counted only once the call has finished
      memset(&one, 0, sizeof one);
      int rc = run_wave(x, &calls[i], 1, nullptr, x->cfg.transitions, &per[i], &one, false, false, nullptr,
                        (uint32_t)i);
      if (rc == HZ_E_OOM && extra) {  // this workspace stops; its call moves on
        per[i].clear();
        std::lock_guard<std::mutex> lock(orphans_mu);
        orphans.push_back(i);
        return HZ_E_OOM;
      }
      if (rc != HZ_OK) {
        stop.store(true);
        return rc;
      }
      add_stats(sx, one);
    }
  };
  std::vector<hz_stats> sts(ws.size());
  for (auto &x : sts) memset(&x, 0, sizeof x);
  std::vector<int> rcs(ws.size(), HZ_OK);
  std::vector<std::string> errs(ws.size());
  std::vector<std::thread> helpers;
  for (size_t j = 1; j < ws.size(); j++) {
    try {
      helpers.emplace_back([&, j] {
        if (cudaSetDevice(ws[j]->device) != cudaSuccess) {
          rcs[j] = HZ_E_CUDA;
          errs[j] = "plain workspace: cudaSetDevice failed";
          stop.store(true);
          return;
        }
        rcs[j] = drive(ws[j], &sts[j], true);
        if (rcs[j] != HZ_OK) errs[j] = g_err;
      });
    } catch (const std::exception &) {  // no thread: its workspace takes no calls, the others take them all
      break;
    }
  }
  rcs[0] = drive(e, &sts[0], false);
  for (auto &t : helpers) t.join();
  if (rcs[0] == HZ_OK && !stop.load()) {
    std::sort(orphans.begin(), orphans.end());
    for (size_t i : orphans) {
      hz_stats one;
      memset(&one, 0, sizeof one);
      rcs[0] = run_wave(e, &calls[i], 1, nullptr, e->cfg.transitions, &per[i], &one, false, false, nullptr,
                        (uint32_t)i);
      if (rcs[0] != HZ_OK) break;
      add_stats(&sts[0], one);
    }
  }
  // the extra workspaces' kernels and profiles count as this engine's
  for (size_t j = 1; j < ws.size(); j++) {
    hz_engine *w = ws[j];
    e->launches += w->launches - launches0[j];
    for (const std::string &name : w->prof_order) {
      if (!e->prof.count(name)) e->prof_order.push_back(name);
      e->prof[name].ms += w->prof[name].ms;
      e->prof[name].n += w->prof[name].n;
    }
    w->prof.clear();
    w->prof_order.clear();
  }
  // a workspace that ran out of device memory gives back what it holds (it
  // is made again on a later pass)
  for (size_t j = ws.size() - 1; j >= 1; j--)
    if (rcs[j] == HZ_E_OOM) {
      auto it = std::find(e->twins.begin(), e->twins.end(), ws[j]);
      if (it != e->twins.end()) e->twins.erase(it);
      hz_engine_destroy(ws[j]);
      cudaGetLastError();
    }
  if (rcs[0] != HZ_OK) return rcs[0];
  for (size_t j = 1; j < ws.size(); j++)
    if (rcs[j] != HZ_OK && rcs[j] != HZ_E_OOM) return fail(rcs[j], "%s", errs[j].c_str());
  for (const hz_stats &x : sts) add_stats(st, x);
  size_t total = 0;
  for (auto &v : per) total += v.size();
  recs->reserve(total);
  for (auto &v : per) recs->insert(recs->end(), v.begin(), v.end());
  return HZ_OK;
}
}  // namespace

// The plain per-chunk form: one wave (launch chain + read-back + host dedup)
// per seed_and_filter call, in the reference's call order.
int hz_run_pass(hz_engine *e, hz_pass_record **out, uint64_t *n, hz_stats *stats) {
  if (!e || !out || !n) return fail(HZ_E_INVALID, "bad argument");
  *out = nullptr;
  *n = 0;
  if (!e->has_query) return fail(HZ_E_STATE, "Engine has no query: swap_query() must be called first");
  if (!e->has_target) return fail(HZ_E_STATE, "no target loaded");
  TRY(set_device(e));
  hz_stats local;
  memset(&local, 0, sizeof local);
  std::vector<HostCall> calls;
  query_calls(e, e->cur_query, &calls);
  std::vector<WaveRecord> recs;
  // (on a caller's stream, every call stays on that stream)
  if (e->plain_streams >= 2 && calls.size() >= 2 && e->st == e->own_st) {
    TRY(run_pass_multi(e, e->plain_streams, calls, &recs, &local));
  } else {
    DeferredDedup defer;  // call i's host dedup runs while call i + 1's kernels do
    for (size_t i = 0; i < calls.size(); i++)
      TRY(run_wave(e, &calls[i], 1, nullptr, e->cfg.transitions, &recs, &local, false, false, &defer, (uint32_t)i));
    defer.finish(e);
  }
  // records of one interval: plus calls before minus calls (call order already)
  if (!recs.empty()) {
    *out = (hz_pass_record *)malloc(recs.size() * sizeof(hz_pass_record));
    if (!*out) return fail(HZ_E_OOM, "host allocation");
    for (size_t i = 0; i < recs.size(); i++)
      (*out)[i] = hz_pass_record{calls[recs[i].call].interval, calls[recs[i].call].strand, recs[i].h};
  }
  *n = recs.size();
  if (stats) *stats = local;
  e->slot[0].kind = 0;
  return HZ_OK;
}

int hz_stage_queries(hz_engine *e, const hz_query *queries, uint32_t nq) {
  if (!e || (nq && !queries)) return fail(HZ_E_INVALID, "null argument");
  std::vector<const uint8_t *> ptrs(nq);
  std::vector<uint64_t> lens(nq);
  for (uint32_t i = 0; i < nq; i++) {
    if (queries[i].len && !queries[i].ascii) return fail(HZ_E_INVALID, "query %u has no bytes", i);
    ptrs[i] = queries[i].ascii;
    lens[i] = queries[i].len;
  }
  TRY(set_device(e));
  return stage_ascii(e, ptrs.data(), lens.data(), nq);
}

int hz_select_query(hz_engine *e, uint32_t index) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  if (index >= e->queries.size()) return fail(HZ_E_INVALID, "query %u not staged (%zu staged)", index, e->queries.size());
  e->cur_query = index;
  e->slot[0].kind = e->slot[1].kind = 0;
  return HZ_OK;
}

// The batched form: the calls of all staged queries, query-major, cut into
// waves of at most wave_positions seed positions at call boundaries.
int hz_run_batched(hz_engine *e, hz_batch_record **out, uint64_t *n, hz_stats *stats) {
  if (!e || !out || !n) return fail(HZ_E_INVALID, "bad argument");
  *out = nullptr;
  *n = 0;
  if (!e->has_query) return fail(HZ_E_STATE, "no query staged");
  if (!e->has_target) return fail(HZ_E_STATE, "no target loaded");
  TRY(set_device(e));
  hz_stats local;
  memset(&local, 0, sizeof local);
  std::vector<HostCall> calls;
  std::vector<WaveRecord> &recs = e->batch_recs;
  recs.clear();
  TRY(run_all_staged(e, &calls, &recs, &local));
  if (!recs.empty()) {
    *out = (hz_batch_record *)malloc(recs.size() * sizeof(hz_batch_record));
    if (!*out) return fail(HZ_E_OOM, "host allocation");
    hz_batch_record *o = *out;
    parallel_ranges(recs.size(), [&](size_t a, size_t b) {
      for (size_t k = a; k < b; k++) {
        const HostCall &c = calls[recs[k].call];
        o[k] = hz_batch_record{c.query, c.interval, c.strand, recs[k].h};
      }
    });
  }
  *n = recs.size();
  if (stats) *stats = local;
  return HZ_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// dedup_and_order of HSPs that already sit in device memory, without
// allocating anything.  Some callers cannot allocate device memory: a host
// program whose own allocator owns the whole device, a serving loop that
// admits work against a fixed memory budget, or a plugin that must not grow
// the process's footprint behind its host's back.  For them this entry point
// runs the batched form's device dedup (radix passes, containment, LASTZ
// order) on a fixed scratch array compiled into this library instead of on
// engine buffers.

namespace {

constexpr uint32_t kNoAllocMax = HZ_NOALLOC_MAX_HSPS;
constexpr uint32_t kNoAllocTiles = (kNoAllocMax + kRadixTile - 1) / kRadixTile;
constexpr uint32_t kNoAllocHist = kNoAllocTiles * kRadixBins;
constexpr uint32_t kNoAllocPartials = kNoAllocHist / kScanTile + 2;
// u32 words: perm_a, perm_b, keys_a, keys_b, dropped flags (kNoAllocMax each),
// radix histograms, scan partials, scan total, kept count
constexpr size_t kNoAllocWords = 5ull * kNoAllocMax + kNoAllocHist + kNoAllocPartials + 2;

}  // namespace

// The scratch: ~6 MB that every GPU which loads this library holds until the
// process exits.  Shared by every call; it keeps the last call's contents.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

namespace {

// Unaligned-tolerant view of hz_segment_pair (the caller's buffers need only
// 4-byte alignment).
struct PlainHsp {
  uint32_t ref_start, query_start, len;
  int32_t score;
};

constexpr int kDroppedField = 6;

__global__ void na_gather_kernel(const PlainHsp *__restrict__ in, const uint32_t *__restrict__ perm,
                                 const uint32_t *__restrict__ dropped, uint32_t n, int field,
                                 uint32_t *__restrict__ keys) {
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t r = perm[i];
    if (field == kDroppedField) {
      keys[i] = dropped[r];
      continue;
    }
    SegmentPair h{in[r].ref_start, in[r].query_start, in[r].len, in[r].score};
    keys[i] = field_key(h, 0u, field);
  }
}

// After the hspComp sort: a record is dropped when it is contained in the
// previous input record (src/hsp.rs:94-126); kept ones are counted.
__global__ void na_flag_kernel(const PlainHsp *__restrict__ in, const uint32_t *__restrict__ perm, uint32_t n,
                               uint32_t *__restrict__ dropped, uint32_t *__restrict__ kept) {
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t r = perm[i];
    bool d = false;
    if (i > 0) {
      const PlainHsp &a = in[perm[i - 1]], &b = in[r];
      d = contained_dev(SegmentPair{a.ref_start, a.query_start, a.len, a.score},
                        SegmentPair{b.ref_start, b.query_start, b.len, b.score});
    }
    dropped[r] = d;
    if (!d) atomicAdd(kept, 1u);
  }
}

__global__ void na_copy_kernel(const PlainHsp *__restrict__ in, const uint32_t *__restrict__ perm,
                               const uint32_t *__restrict__ kept, PlainHsp *__restrict__ out,
                               uint32_t *__restrict__ n_out) {
  const uint32_t k = *kept;
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += stride) out[i] = in[perm[i]];
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = k;
}

// The unique id of the calling thread's current CUDA context (0 if there is
// none or the driver cannot say).  Ids are never reused within a process, so
// a context torn down and created again (cudaDeviceReset) gets a new one.
unsigned long long current_context_id() {
  typedef CUresult (*GetCurrentFn)(CUcontext *);
  typedef CUresult (*GetIdFn)(CUcontext, unsigned long long *);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetIdFn>(p);
    cudaGetLastError();
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

// The scratch's device address, looked up with the device current (host
// code cannot use the symbol itself as a device pointer) the first time a
// context of that device calls, and again whenever the device's context has
// changed since -- after a cudaDeviceReset the old address is dead.
int noalloc_scratch(int device, uint32_t **out) {
  static uint32_t *addr[64] = {nullptr};
  static unsigned long long ctx_of[64] = {0};
  static std::mutex mu;
  if (device < 0 || device >= 64) return fail(HZ_E_INVALID, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(mu);
  const unsigned long long ctx = current_context_id();
  if (!addr[device] || ctx == 0 || ctx != ctx_of[device]) {
    void *p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess) return fail(HZ_E_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(err));
    addr[device] = static_cast<uint32_t *>(p);
    ctx_of[device] = current_context_id();  // the lookup may have created the context
  }
  *out = addr[device];
  return HZ_OK;
}

// [a, a + na) and [b, b + nb) share a byte
bool overlaps(const void *a, size_t na, const void *b, size_t nb) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return na && nb && x < y + nb && y < x + na;
}

}  // namespace

extern "C" {

int hz_dedup_and_order_device_noalloc(const hz_segment_pair *d_in, uint32_t n, hz_segment_pair *d_out,
                                      uint32_t *d_n_out, void *stream) {
  if (n > kNoAllocMax)
    return fail(HZ_E_INVALID, "%u HSPs exceed the %u that this entry point's fixed scratch holds", n, kNoAllocMax);
  if (!d_n_out || (n && (!d_in || !d_out))) return fail(HZ_E_INVALID, "null device pointer");
  if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out) |
       reinterpret_cast<uintptr_t>(d_n_out)) & 3)
    return fail(HZ_E_INVALID, "device buffers must be 4-byte aligned");
  // the kernels read d_in while they write d_out and d_n_out, so the three
  // must be disjoint (no in-place dedup)
  const size_t bytes = (size_t)n * sizeof(hz_segment_pair);
  if (overlaps(d_in, bytes, d_out, bytes) || overlaps(d_n_out, 4, d_in, bytes) || overlaps(d_n_out, 4, d_out, bytes))
    return fail(HZ_E_INVALID, "d_in, d_out and d_n_out must not overlap");
  int device = 0;
  CK(cudaGetDevice(&device));
  uint32_t *base = nullptr;
  TRY(noalloc_scratch(device, &base));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t *perm_a = base, *perm_b = perm_a + kNoAllocMax, *keys_a = perm_b + kNoAllocMax,
           *keys_b = keys_a + kNoAllocMax, *dropped = keys_b + kNoAllocMax, *hist = dropped + kNoAllocMax,
           *partials = hist + kNoAllocHist, *total = partials + kNoAllocPartials, *kept = total + 1;
  // the kept count accumulates and must start at zero; everything else is
  // fully rewritten before it is read
  CK(cudaMemsetAsync(kept, 0, 4, s));
  const PlainHsp *in = reinterpret_cast<const PlainHsp *>(d_in);
  const unsigned g = grid_for(n, 256, 1024);
  iota_kernel<<<g, 256, 0, s>>>(perm_a, n);
  const uint64_t tiles = (n + kRadixTile - 1) / kRadixTile;
  auto sort_by = [&](const int *fields, int nf) {
    for (int fi = 0; fi < nf; fi++) {
      const int f = fields[fi];
      na_gather_kernel<<<g, 256, 0, s>>>(in, perm_a, dropped, n, f, keys_a);
      const int passes = f == kDroppedField ? 1 : 4;
      for (int p = 0; p < passes && n; p++) {
        radix_hist_kernel<<<(unsigned)tiles, kRadixThreads, 0, s>>>(keys_a, n, 8 * p, hist, tiles);
        exclusive_scan<uint32_t>(hist, hist, tiles * kRadixBins, partials, total, s);
        radix_scatter_kernel<<<(unsigned)tiles, kRadixThreads, 0, s>>>(keys_a, perm_a, n, 8 * p, hist, tiles,
                                                                      keys_b, perm_b);
        std::swap(keys_a, keys_b);
        std::swap(perm_a, perm_b);
      }
    }
  };
  static const int by_diagonal_key[4] = {kScoreDesc, kLen, kRefStart, kDiag};
  // dropped records last, the kept ones in LASTZ order first
  static const int by_lastz_key[5] = {kScoreDesc, kLen, kRefStart, kQueryStart, kDroppedField};
  if (n) {
    sort_by(by_diagonal_key, 4);
    na_flag_kernel<<<g, 256, 0, s>>>(in, perm_a, n, dropped, kept);
    sort_by(by_lastz_key, 5);
  }
  na_copy_kernel<<<g, 256, 0, s>>>(in, perm_a, kept, reinterpret_cast<PlainHsp *>(d_out), d_n_out);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return fail(HZ_E_CUDA, "dedup launch: %s", cudaGetErrorString(err));
  return HZ_OK;
}

int hz_render_records(const hz_segment_record *recs, uint64_t n, const char *const *r_names, uint32_t nr,
                      const char *const *q_names, uint32_t nq, char strand, char **out, uint64_t *out_len) {
  if (!out || !out_len || (n && (!recs || !r_names || !q_names))) return fail(HZ_E_INVALID, "null argument");
  *out = nullptr;
  *out_len = 0;
  std::vector<size_t> rl(nr), ql(nq);
  for (uint32_t i = 0; i < nr; i++) rl[i] = r_names[i] ? strlen(r_names[i]) : 0;
  for (uint32_t i = 0; i < nq; i++) ql[i] = q_names[i] ? strlen(q_names[i]) : 0;
  // exact size first: names + up to 20 digits per number + separators
  uint64_t cap = 1;
  for (uint64_t i = 0; i < n; i++) {
    if (recs[i].r_chr >= nr || recs[i].q_chr >= nq)
      return fail(HZ_E_INVALID, "record %llu names chromosome (%u, %u) outside the tables (%u, %u)",
                  (unsigned long long)i, recs[i].r_chr, recs[i].q_chr, nr, nq);
    cap += rl[recs[i].r_chr] + ql[recs[i].q_chr] + 5 * 20 + 11 + 8;
  }
  char *buf = (char *)malloc(cap);
  if (!buf) return fail(HZ_E_OOM, "host allocation of %llu bytes", (unsigned long long)cap);
  char *w = buf;
  auto num = [&](unsigned long long v) {
    char tmp[24];
    int k = 0;
    do {
      tmp[k++] = (char)('0' + v % 10);
      v /= 10;
    } while (v);
    while (k) *w++ = tmp[--k];
  };
  for (uint64_t i = 0; i < n; i++) {
    const hz_segment_record &r = recs[i];
    memcpy(w, r_names[r.r_chr], rl[r.r_chr]);
    w += rl[r.r_chr];
    *w++ = '\t';
    num(r.r_start);
    *w++ = '\t';
    num(r.r_end);
    *w++ = '\t';
    memcpy(w, q_names[r.q_chr], ql[r.q_chr]);
    w += ql[r.q_chr];
    *w++ = '\t';
    num(r.q_start);
    *w++ = '\t';
    num(r.q_end);
    *w++ = '\t';
    *w++ = strand;
    *w++ = '\t';
    if (r.score < 0) {
      *w++ = '-';
      num((unsigned long long)(-(long long)r.score));
    } else {
      num((unsigned long long)r.score);
    }
    *w++ = '\n';
  }
  *w = 0;
  *out = buf;
  *out_len = (uint64_t)(w - buf);
  return HZ_OK;
}

int hz_dedup_and_order(hz_segment_pair *h, uint64_t n, uint64_t *n_out) {
  if ((n && !h) || !n_out) return fail(HZ_E_INVALID, "null argument");
  *n_out = dedup_and_order(h, n);
  return HZ_OK;
}

int hz_engine_set_profiling(hz_engine *e, int on) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  TRY(e->sync());
  e->profiling = on != 0;
  return HZ_OK;
}

int hz_engine_profile_entry(hz_engine *e, uint32_t i, char *name, uint32_t name_cap, double *ms, uint64_t *launches) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  TRY(e->sync());
  if (i >= e->prof_order.size()) return HZ_E_INVALID;
  const std::string &k = e->prof_order[i];
  if (name && name_cap) {
    strncpy(name, k.c_str(), name_cap - 1);
    name[name_cap - 1] = 0;
  }
  if (ms) *ms = e->prof[k].ms;
  if (launches) *launches = e->prof[k].n;
  return HZ_OK;
}

int hz_engine_profile_reset(hz_engine *e) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  TRY(e->sync());
  e->prof.clear();
  e->prof_order.clear();
  return HZ_OK;
}

uint64_t hz_engine_launches(hz_engine *e) {
  if (!e) return 0;
  return e->launches + (e->server ? server_launches(e->server) : 0);
}

int hz_engine_set_tuning(hz_engine *e, const char *key, int64_t value) {
  if (!e || !key) return fail(HZ_E_INVALID, "null argument");
  std::string k(key);
  if (k == "gate_tile") {
    if (value != 64 && value != 128 && value != 256)
      return fail(HZ_E_INVALID, "gate_tile must be 64, 128 or 256");
    e->gate_tile = (int)value;
  } else if (k == "gate_version") {
    if (value != 1 && value != 2) return fail(HZ_E_INVALID, "gate_version must be 1 or 2");
    e->gate_version = (int)value;
  } else if (k == "gate_sparse") {
    if (value < -1 || value > 1) return fail(HZ_E_INVALID, "gate_sparse must be -1, 0 or 1");
    e->gate_sparse = (int)value;
  } else if (k == "gate_cap") {
    if (value < 8 || value > 65528 || value % 8) return fail(HZ_E_INVALID, "gate_cap must be a multiple of 8 in 8..65528");
    e->gate_cap = (uint32_t)value;
  } else if (k == "gate_blocks_per_sm") {
    if (value < 0 || value > 32) return fail(HZ_E_INVALID, "gate_blocks_per_sm must be 0..32");
    e->gate_blocks_per_sm = (int)value;
  } else if (k == "device_dedup") {
    e->device_dedup = value != 0;
  } else if (k == "device_dedup_min") {
    if (value < 1 || value > 0xFFFFFFFFll) return fail(HZ_E_INVALID, "device_dedup_min must be 1..2^32-1");
    e->device_dedup_min = (uint32_t)value;
  } else if (k == "graph") {
    e->use_graph = value != 0;
  } else if (k == "wave_positions") {
    if (value < 1 || value >= (1ll << 31)) return fail(HZ_E_INVALID, "wave_positions must be 1..2^31-1");
    e->wave_positions = (uint64_t)value;
  } else if (k == "wave_hits_cap") {
    if (value < (1ll << 20)) return fail(HZ_E_INVALID, "wave_hits_cap must be at least 2^20");
    e->wave_hits_cap = (uint64_t)value;
  } else if (k == "plain_streams") {
    if (value < 1 || value > 4) return fail(HZ_E_INVALID, "plain_streams must be 1..4");
    e->plain_streams = (int)value;
    // workspaces beyond the new count give their wave buffers back
    while ((int)e->twins.size() > e->plain_streams - 1) {
      hz_engine_destroy(e->twins.back());
      e->twins.pop_back();
    }
  } else if (k == "tile_cap" || k == "cand_cap" || k == "raw_cap") {
    // starting capacities; a wave that needs more grows them and runs again
    if (value < 16 || value > 0x7FFFFFFFll) return fail(HZ_E_INVALID, "%s must be 16..2^31-1", key);
    (k == "tile_cap" ? e->tile_cap : k == "cand_cap" ? e->cand_cap : e->raw_cap) = (uint32_t)value;
  } else {
    return fail(HZ_E_INVALID, "unknown tuning key %s", key);
  }
  return HZ_OK;
}

int hz_engine_autotune(hz_engine *e, uint64_t sample_positions, hz_tuning *out) {
  if (!e || !out) return fail(HZ_E_INVALID, "null argument");
  if (!e->has_target) return fail(HZ_E_STATE, "no target loaded");
  if (e->queries.empty()) return fail(HZ_E_STATE, "no staged queries to tune on");
  TRY(set_device(e));
  if (sample_positions == 0) sample_positions = 1ull << 24;
  // sample: every k-th call of the staged work, so that the sample spans
  // the queries' length mix, up to sample_positions seed positions
  std::vector<HostCall> all, sample;
  for (uint32_t q = 0; q < e->queries.size(); q++) query_calls(e, q, &all);
  if (all.empty()) return fail(HZ_E_STATE, "the staged queries have no seed positions");
  uint64_t total = 0;
  for (auto &c : all) total += c.end - c.start;
  uint64_t stride = std::max<uint64_t>(1, total / sample_positions);
  uint64_t got = 0;
  for (size_t i = 0; i < all.size() && got < sample_positions; i += stride) {
    sample.push_back(all[i]);
    got += all[i].end - all[i].start;
  }
  struct Knobs {
    int tile;
    uint32_t cap;
    bool graph;
  };
  const Knobs start{e->gate_tile, e->gate_cap, e->use_graph};
  std::vector<Knobs> cands;
  for (int tile : {64, 128, 256})
    for (uint32_t cap : {64u, 128u, 256u, 512u, 1024u})
      for (bool graph : {false, true}) cands.push_back(Knobs{tile, cap, graph});
  bool prof = e->profiling;
  e->profiling = false;
  auto time_once = [&](const Knobs &k, double *ms) -> int {
    e->gate_tile = k.tile;
    e->gate_cap = k.cap;
    e->use_graph = k.graph;
    std::vector<HostCall> calls(sample);
    std::vector<WaveRecord> recs;
    TRY(e->sync());
    auto t0 = std::chrono::steady_clock::now();
    TRY(run_calls(e, &calls, &recs, nullptr));
    TRY(e->sync());
    *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return HZ_OK;
  };
  double best = 1e300, at_start = 0;
  Knobs pick = start;
  int rc = HZ_OK;
  {
    double warm;
    rc = time_once(start, &warm);  // first touch: buffer growth, graph instantiation
    if (rc == HZ_OK) rc = time_once(start, &at_start);
    best = at_start;
  }
  for (size_t i = 0; i < cands.size() && rc == HZ_OK; i++) {
    double a = 0, b = 0;
    rc = time_once(cands[i], &a);
    if (rc == HZ_OK) rc = time_once(cands[i], &b);
    double m = std::min(a, b);
    if (rc == HZ_OK && m < best) {
      best = m;
      pick = cands[i];
    }
  }
  e->profiling = prof;
  e->gate_tile = pick.tile;
  e->gate_cap = pick.cap;
  e->use_graph = pick.graph;
  if (rc != HZ_OK) {
    e->gate_tile = start.tile;
    e->gate_cap = start.cap;
    e->use_graph = start.graph;
    return rc;
  }
  out->gate_tile = pick.tile;
  out->gate_cap = (int32_t)pick.cap;
  out->gate_blocks_per_sm = e->gate_blocks_per_sm;
  out->graph = pick.graph ? 1 : 0;
  out->best_ms = best;
  out->start_ms = at_start;
  out->candidates = (uint32_t)cands.size();
  out->sample_calls = (uint32_t)sample.size();
  out->sample_positions = got;
  return HZ_OK;
}

int hz_engine_set_stream(hz_engine *e, void *stream) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  TRY(set_device(e));
  TRY(e->sync());
  e->st = stream ? (cudaStream_t)stream : e->own_st;
  return HZ_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving loop.  The engine's target stays resident; worker threads, each
// with its own workspace (query store, wave buffers, stream) over the shared
// target tables, keep taking the queued requests that fit the memory budget
// and run them as one batched pass.  A request that arrives while others are
// on the GPU joins the next batch a worker forms, so requests are admitted as
// workers and memory free up, and the batches of different workers overlap on
// the device.  A request's records equal what hz_run_pass returns for its
// query alone (tests/test_gpu_serving.py).

enum ServeState { kPending = 0, kRunning = 1, kDone = 2, kCancelled = 3, kFailed = 4 };

struct ServeRequest {
  uint64_t ticket = 0;
  std::vector<uint8_t> ascii;
  int state = kPending;
  int err = HZ_OK;
  std::string msg;
  std::vector<hz_pass_record> recs;
  uint32_t batch_queries = 0, worker = 0;
  std::chrono::steady_clock::time_point t_submit, t_admit, t_done;
};

struct Server {
  hz_engine *owner = nullptr;
  std::vector<hz_engine *> workers;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> pending;
  std::unordered_map<uint64_t, std::shared_ptr<ServeRequest>> reqs;
  uint64_t next_ticket = 1;
  // Device memory against the budget: per worker, the bytes it holds while
  // idle (its measured buffers) or, while it runs a batch, the larger of
  // those and the batch's estimate; in_flight is their sum.
  uint64_t budget = 0, in_flight = 0;
  std::vector<uint64_t> reserved;
  // rates the estimates use: hits per seed position, candidates and raw HSPs
  // per hit -- the largest seen so far, starting from the target's average
  // and 1e-3
  double hits_per_pos = 0, cand_per_hit = 1e-3, raw_per_hit = 1e-3;
  int gate_tile = 128;
  // bumped by a worker whose head request cannot fit while nothing runs:
  // idle workers then give their buffers back
  uint64_t trim_epoch = 0;
  uint32_t max_batch = 64;
  bool stopping = false;
  hz_stats totals{};
  uint64_t running = 0;
  uint64_t launches = 0;  // kernel launches of the workers
};

uint64_t server_launches(Server *s) {
  std::lock_guard<std::mutex> lock(s->mu);
  return s->launches;
}

namespace {

template <typename T> uint64_t dbytes(const DBuf<T> &b) { return b.p ? b.cap * sizeof(T) + 64 : 0; }

// Device bytes an engine's own working buffers hold: its query store (unless
// it borrows another engine's) and every wave and dedup buffer.
uint64_t wave_footprint(const hz_engine *w) {
  uint64_t b = w->aliases_query ? 0 : dbytes(w->qstore.buf) + dbytes(w->qry_p.blk);
  b += dbytes(w->qascii) + dbytes(w->calls) + dbytes(w->pos_hits) + dbytes(w->np_pos) + dbytes(w->call_nz_lo) +
       dbytes(w->pos_kmer) + dbytes(w->np_kmer) +
       dbytes(w->scope_call) + dbytes(w->raw_scope) + dbytes(w->tile_first) + dbytes(w->tile_call) +
       dbytes(w->np_excl) + dbytes(w->call_hit_lo) + dbytes(w->scope_lo) + dbytes(w->np_partial) +
       dbytes(w->np_grand) + dbytes(w->tot) + dbytes(w->cand) + dbytes(w->raw) + dbytes(w->d_out);
  for (const DBuf<uint32_t> *x : {&w->d_perm_a, &w->d_perm_b, &w->d_keys_a, &w->d_keys_b, &w->d_keep,
                                  &w->d_keep_excl, &w->d_hist, &w->d_hpart, &w->d_total})
    b += dbytes(*x);
  return b;
}

// Gives an idle serving worker's query store, wave and dedup buffers back
// (they grow again on its next batch, which restages its queries anyway).
void release_wave_buffers(hz_engine *w) {
  cudaStreamSynchronize(w->st);
  if (!w->aliases_query) {
    w->qstore.buf.release();
    w->qry_p.release();
  }
  w->qascii.release();
  for (DBuf<uint32_t> *x : {&w->pos_hits, &w->np_pos, &w->call_nz_lo, &w->scope_call, &w->raw_scope, &w->tile_first,
                            &w->tile_call, &w->pos_kmer, &w->np_kmer, &w->d_perm_a, &w->d_perm_b, &w->d_keys_a, &w->d_keys_b, &w->d_keep,
                            &w->d_keep_excl, &w->d_hist, &w->d_hpart, &w->d_total})
    x->release();
  w->np_excl.release();
  w->call_hit_lo.release();
  w->scope_lo.release();
  w->np_partial.release();
  w->np_grand.release();
  w->cand.release();
  w->raw.release();
  w->d_out.release();
  w->calls.release();
  w->tot.release();
}

// Device working memory a request of `len` bases is expected to need while
// it runs: both strands of the query store (1 B per base, and 1 B for its
// packed copy) and of the per-position counts, k-mers and compaction (24 B
// per position), plus the hit-dependent buffers -- the gate's tile table (8 B
// per tile of hits), candidates (32 B each), raw HSPs (20 B each) and their
// dedup scratch (24 B each) -- at the server's current rates.
uint64_t serve_estimate(const Server *s, uint64_t len) {
  const double pos = 2.0 * (double)len;
  const double hits = pos * s->hits_per_pos;
  const double per_hit = 8.0 / s->gate_tile + 32.0 * s->cand_per_hit + 44.0 * s->raw_per_hit;
  return (uint64_t)(pos * (2 + 24) + hits * per_hit) + (1ull << 20);
}

// Copies into `w` what a workspace shares with `e`: the resident target
// tables (borrowed, not owned), the configuration and the launch knobs.
void share_target(hz_engine *w, const hz_engine *e) {
  w->device = e->device;
  w->sm_count = e->sm_count;
  w->cfg = e->cfg;
  w->shape = e->shape;
  w->max_hits = e->max_hits;
  w->ref.buf.p = e->ref.buf.p;
  w->ref.buf.cap = e->ref.buf.cap;
  w->ref.len = e->ref.len;
  w->rlen = e->rlen;
  w->index_table.p = e->index_table.p;
  w->index_table.cap = e->index_table.cap;
  w->index_len = e->index_len;
  w->pos_table.p = e->pos_table.p;
  w->pos_table.cap = e->pos_table.cap;
  w->nbr_hits.p = e->nbr_hits.p;
  w->nbr_hits.cap = e->nbr_hits.cap;
  w->has_nbr = e->has_nbr;
  w->n_pos = e->n_pos;
  w->ref_p = e->ref_p;
  w->has_target = true;
  w->owns_target = false;
  w->gate_version = e->gate_version;
  w->gate_sparse = e->gate_sparse;
  w->gate_tile = e->gate_tile;
  w->gate_cap = e->gate_cap;
  w->gate_blocks_per_sm = e->gate_blocks_per_sm;
  w->wave_positions = e->wave_positions;
  w->wave_hits_cap = e->wave_hits_cap;
  w->device_dedup = e->device_dedup;
  w->device_dedup_min = e->device_dedup_min;
  w->use_graph = e->use_graph;
  // starting capacities: at least the owner's (its hints and what its waves
  // have grown to), keeping what the workspace has grown to itself
  w->tile_cap = std::max(w->tile_cap, e->tile_cap);
  w->cand_cap = std::max(w->cand_cap, e->cand_cap);
  w->raw_cap = std::max(w->raw_cap, e->raw_cap);
}

// A workspace that shares `e`'s resident target tables without owning them.
int clone_shared(hz_engine *e, hz_engine **out) {
  hz_engine *w = new hz_engine();
  share_target(w, e);
  cudaError_t err = cudaStreamCreateWithFlags(&w->own_st, cudaStreamNonBlocking);
  if (err != cudaSuccess) {
    w->owns_target = false;
    delete w;
    return fail(HZ_E_CUDA, "worker stream: %s", cudaGetErrorString(err));
  }
  w->st = w->own_st;
  int rc = w->qstore.ensure(0, w->st);
  if (rc != HZ_OK) {
    hz_engine_destroy(w);
    return rc;
  }
  *out = w;
  return HZ_OK;
}

// The request behind a queued ticket, or null once it was cancelled (and
// perhaps already polled, which drops it from the ticket map).
std::shared_ptr<ServeRequest> queued_request(Server *s, uint64_t ticket) {
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end() || it->second->state != kPending) return nullptr;
  return it->second;
}

// One batched pass of `qs` on worker `w`: the records of request k go to
// (*out)[k].  Returns the pass's status.
int serve_pass(hz_engine *w, const std::vector<std::shared_ptr<ServeRequest>> &qs,
               std::vector<std::vector<hz_pass_record>> *out, hz_stats *st) {
  std::vector<const uint8_t *> ptrs;
  std::vector<uint64_t> lens;
  for (auto &r : qs) {
    ptrs.push_back(r->ascii.data());
    lens.push_back(r->ascii.size());
  }
  std::vector<HostCall> calls;
  std::vector<WaveRecord> recs;
  out->assign(qs.size(), {});
  TRY(stage_ascii(w, ptrs.data(), lens.data(), (uint32_t)qs.size()));
  TRY(run_all_staged(w, &calls, &recs, st));
  for (auto &wr : recs) {
    const HostCall &c = calls[wr.call];
    (*out)[c.query].push_back(hz_pass_record{c.interval, c.strand, wr.h});
  }
  return HZ_OK;
}

void serve_worker(Server *s, uint32_t index, hz_engine *w) {
  cudaSetDevice(w->device);
  uint64_t seen_epoch = 0;
  while (true) {
    std::vector<std::shared_ptr<ServeRequest>> batch;
    bool trim = false;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      while (true) {
        while (!s->pending.empty() && !queued_request(s, s->pending.front())) s->pending.pop_front();
        if (s->stopping && s->pending.empty()) return;
        if (s->trim_epoch != seen_epoch) {  // some request waits for idle buffers
          seen_epoch = s->trim_epoch;
          if (s->reserved[index]) {
            trim = true;
            break;
          }
        }
        // admit queued requests, in arrival order, while this worker's
        // reservation -- its own buffers or the batch's estimate, whichever
        // is larger -- fits the budget beside every other worker's
        const uint64_t others = s->in_flight - s->reserved[index];
        uint64_t want = 0;
        while (!s->pending.empty() && batch.size() < s->max_batch) {
          auto r = queued_request(s, s->pending.front());
          if (!r) {
            s->pending.pop_front();
            continue;
          }
          const uint64_t est = serve_estimate(s, r->ascii.size());
          // (a request alone on an otherwise empty device always runs: its
          // estimate may have outgrown the budget since it was submitted)
          const bool alone = batch.empty() && others == 0;
          if (!alone && others + std::max(s->reserved[index], want + est) > s->budget) break;
          s->pending.pop_front();
          r->state = kRunning;
          r->t_admit = std::chrono::steady_clock::now();
          want += est;
          s->running += 1;
          batch.push_back(r);
        }
        if (!batch.empty()) {
          const uint64_t res = std::max(s->reserved[index], want);
          s->in_flight += res - s->reserved[index];
          s->reserved[index] = res;
          break;
        }
        if (!s->pending.empty()) {
          if (s->reserved[index]) {  // the head does not fit: first give back this worker's own buffers
            trim = true;
            break;
          }
          if (s->running == 0) {  // nothing will finish: ask the idle workers for theirs
            s->trim_epoch++;
            seen_epoch = s->trim_epoch;
            s->cv_work.notify_all();
          }
        }
        s->cv_work.wait(lock);
      }
    }
    if (trim) {
      release_wave_buffers(w);
      {
        std::lock_guard<std::mutex> lock(s->mu);
        const uint64_t fp = wave_footprint(w);
        s->in_flight = s->in_flight - s->reserved[index] + fp;
        s->reserved[index] = fp;
      }
      s->cv_work.notify_all();
      continue;
    }
    // one batched pass over the admitted queries; if it fails, each request
    // runs again alone, so only the ones that fail by themselves report it
    std::vector<std::vector<hz_pass_record>> recs;
    std::vector<int> rcs(batch.size(), HZ_OK);
    std::vector<std::string> msgs(batch.size());
    hz_stats st{};
    uint64_t l0 = w->launches, c0 = w->cand_seen;
    int rc = serve_pass(w, batch, &recs, &st);
    if (rc != HZ_OK && batch.size() > 1) {
      st = hz_stats{};
      c0 = w->cand_seen;
      recs.assign(batch.size(), {});
      for (size_t k = 0; k < batch.size(); k++) {
        std::vector<std::vector<hz_pass_record>> one;
        hz_stats s1{};
        rcs[k] = serve_pass(w, {batch[k]}, &one, &s1);
        if (rcs[k] == HZ_OK) {
          recs[k] = std::move(one[0]);
          add_stats(&st, s1);
        } else {
          msgs[k] = g_err;
        }
      }
    } else if (rc != HZ_OK) {
      rcs[0] = rc;
      msgs[0] = g_err;
    }
    const uint64_t fp = wave_footprint(w);
    bool over = false;
    {
      std::lock_guard<std::mutex> lock(s->mu);
      auto now = std::chrono::steady_clock::now();
      uint64_t positions = 0;
      for (size_t k = 0; k < batch.size(); k++) {
        auto &r = batch[k];
        if (rcs[k] == HZ_OK) positions += 2 * r->ascii.size();
        r->recs = std::move(recs[k]);
        r->state = rcs[k] == HZ_OK ? kDone : kFailed;
        r->err = rcs[k];
        r->msg = msgs[k];
        r->batch_queries = (uint32_t)batch.size();
        r->worker = index;
        r->t_done = now;
        r->ascii.clear();
        r->ascii.shrink_to_fit();
        s->running -= 1;
      }
      // what this worker holds now replaces the batch's reservation
      s->in_flight = s->in_flight - s->reserved[index] + fp;
      s->reserved[index] = fp;
      over = s->in_flight > s->budget;
      if (positions && st.hits) {
        s->hits_per_pos = std::max(s->hits_per_pos, (double)st.hits / (double)positions);
        s->cand_per_hit = std::max(s->cand_per_hit, (double)(w->cand_seen - c0) / (double)st.hits);
        s->raw_per_hit = std::max(s->raw_per_hit, (double)st.raw_hsps / (double)st.hits);
      }
      s->launches += w->launches - l0;
      s->totals.seeds += st.seeds;
      s->totals.hits += st.hits;
      s->totals.raw_hsps += st.raw_hsps;
      s->totals.hsps += st.hsps;
      s->totals.cells += st.cells;
      s->totals.calls += st.calls;
    }
    if (over) {  // the batch outgrew its estimate: give the buffers back now
      release_wave_buffers(w);
      std::lock_guard<std::mutex> lock(s->mu);
      const uint64_t left = wave_footprint(w);
      s->in_flight = s->in_flight - s->reserved[index] + left;
      s->reserved[index] = left;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

}  // namespace

extern "C" {

int hz_serve_start(hz_engine *e, const hz_serve_config *cfg) {
  if (!e || !cfg) return fail(HZ_E_INVALID, "null argument");
  if (e->server) return fail(HZ_E_STATE, "the serving loop is already running");
  if (!e->has_target) return fail(HZ_E_STATE, "no target loaded");
  if (cfg->workers < 1 || cfg->workers > 8) return fail(HZ_E_INVALID, "workers must be 1..8");
  if (cfg->budget_bytes == 0) return fail(HZ_E_INVALID, "budget_bytes must be > 0");
  TRY(set_device(e));
  TRY(e->sync());
  Server *s = new Server();
  s->owner = e;
  s->budget = cfg->budget_bytes;
  s->max_batch = cfg->max_batch_queries ? cfg->max_batch_queries : 64;
  for (uint32_t i = 0; i < cfg->workers; i++) {
    hz_engine *w = nullptr;
    int rc = clone_shared(e, &w);
    if (rc != HZ_OK) {
      for (auto *x : s->workers) hz_engine_destroy(x);
      delete s;
      return rc;
    }
    s->workers.push_back(w);
  }
  s->reserved.assign(s->workers.size(), 0);
  for (size_t i = 0; i < s->workers.size(); i++) {
    s->reserved[i] = wave_footprint(s->workers[i]);
    s->in_flight += s->reserved[i];
  }
  // starting rate: a query k-mer drawn uniformly meets per_pos buckets of the
  // average size
  s->hits_per_pos = e->index_len ? (double)e->per_pos(e->cfg.transitions) * (double)e->n_pos / (double)e->index_len : 0;
  s->gate_tile = e->gate_tile;
  e->server = s;
  for (uint32_t i = 0; i < (uint32_t)s->workers.size(); i++) s->threads.emplace_back(serve_worker, s, i, s->workers[i]);
  return HZ_OK;
}

int hz_serve_submit(hz_engine *e, const uint8_t *ascii, uint64_t len, uint64_t *ticket) {
  if (!e || !ticket || (len && !ascii)) return fail(HZ_E_INVALID, "null argument");
  Server *s = e->server;
  if (!s) return fail(HZ_E_STATE, "the serving loop is not running");
  if (len > 0xFFFFFFFFull) return fail(HZ_E_INVALID, "query block exceeds u32 coordinates");
  auto r = std::make_shared<ServeRequest>();
  r->t_submit = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stopping) return fail(HZ_E_STATE, "the serving loop is stopping");
    const uint64_t est = serve_estimate(s, len);
    if (est > s->budget)
      return fail(HZ_E_BUDGET, "a %llu-base query needs ~%llu bytes of working memory, above the %llu-byte budget",
                  (unsigned long long)len, (unsigned long long)est, (unsigned long long)s->budget);
    r->ascii.assign(ascii, ascii + len);
    r->ticket = s->next_ticket++;
    s->reqs[r->ticket] = r;
    s->pending.push_back(r->ticket);
  }
  s->cv_work.notify_one();
  *ticket = r->ticket;
  return HZ_OK;
}

int hz_serve_poll(hz_engine *e, uint64_t ticket, int timeout_ms, hz_pass_record **out, uint64_t *n,
                  hz_serve_times *times) {
  if (!e || !out || !n) return fail(HZ_E_INVALID, "null argument");
  *out = nullptr;
  *n = 0;
  Server *s = e->server;
  if (!s) return fail(HZ_E_STATE, "the serving loop is not running");
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(HZ_E_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
  auto r = it->second;
  auto done = [&] { return r->state == kDone || r->state == kFailed || r->state == kCancelled; };
  if (!done()) {
    if (timeout_ms < 0) s->cv_done.wait(lock, done);
    else if (!s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), done))
      return fail(HZ_E_TIMEOUT, "ticket %llu still %s", (unsigned long long)ticket,
                  r->state == kPending ? "queued" : "running");
  }
  s->reqs.erase(it);
  if (times) {
    auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
      return std::chrono::duration<double, std::milli>(b - a).count();
    };
    times->queued_ms = r->state == kCancelled ? 0.0 : ms(r->t_submit, r->t_admit);
    times->service_ms = r->state == kCancelled ? 0.0 : ms(r->t_admit, r->t_done);
    times->total_ms = r->state == kCancelled ? 0.0 : ms(r->t_submit, r->t_done);
    times->batch_queries = r->batch_queries;
    times->worker = r->worker;
  }
  if (r->state == kCancelled) return fail(HZ_E_STATE, "ticket %llu was cancelled", (unsigned long long)ticket);
  if (r->state == kFailed) return fail(r->err, "%s", r->msg.c_str());
  if (!r->recs.empty()) {
    *out = (hz_pass_record *)malloc(r->recs.size() * sizeof(hz_pass_record));
    if (!*out) return fail(HZ_E_OOM, "host allocation");
    memcpy(*out, r->recs.data(), r->recs.size() * sizeof(hz_pass_record));
  }
  *n = r->recs.size();
  return HZ_OK;
}

int hz_serve_estimate(hz_engine *e, uint64_t len, uint64_t *bytes) {
  if (!e || !bytes) return fail(HZ_E_INVALID, "null argument");
  Server *s = e->server;
  if (!s) return fail(HZ_E_STATE, "the serving loop is not running");
  std::lock_guard<std::mutex> lock(s->mu);
  *bytes = serve_estimate(s, len);
  return HZ_OK;
}

int hz_serve_stats(hz_engine *e, hz_stats *stats, uint64_t *queued, uint64_t *running) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  Server *s = e->server;
  if (!s) return fail(HZ_E_STATE, "the serving loop is not running");
  std::lock_guard<std::mutex> lock(s->mu);
  if (stats) *stats = s->totals;
  if (queued) {
    uint64_t q = 0;
    for (uint64_t t : s->pending)
      if (queued_request(s, t)) q++;
    *queued = q;
  }
  if (running) *running = s->running;
  return HZ_OK;
}

int hz_serve_cancel(hz_engine *e, uint64_t ticket) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  Server *s = e->server;
  if (!s) return fail(HZ_E_STATE, "the serving loop is not running");
  {
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(HZ_E_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    if (it->second->state != kPending)
      return fail(HZ_E_STATE, "ticket %llu is already running or finished", (unsigned long long)ticket);
    it->second->state = kCancelled;
  }
  s->cv_done.notify_all();
  s->cv_work.notify_all();
  return HZ_OK;
}

int hz_serve_stop(hz_engine *e) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  Server *s = e->server;
  if (!s) return HZ_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto &t : s->threads) t.join();
  for (auto *w : s->workers) hz_engine_destroy(w);
  {
    std::lock_guard<std::mutex> lock(s->mu);
    for (auto &kv : s->reqs)
      if (kv.second->state == kPending) kv.second->state = kCancelled;
  }
  s->cv_done.notify_all();
  e->launches += s->launches;
  e->server = nullptr;
  delete s;
  return HZ_OK;
}

}  // extern "C"
