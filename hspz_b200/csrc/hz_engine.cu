// Host side of the B200 seed-and-filter engine and its C ABI
// (include/hspz_b200.h).  One engine = one device, one stream, resident
// target tables, the swapped-in query and two seed slots, mirroring the
// reference's Engine (src/gpu/mod.rs:817-2307).
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/hspz_b200.h"
#include "hz_kernels.cuh"
#include "hz_scan.cuh"

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

#define TRY(x)                \
  do {                        \
    int r_ = (x);             \
    if (r_ != HZ_OK) return r_; \
  } while (0)

// Grow-only device buffer.  Growing waits for the stream, because a queued
// kernel may still read the old allocation.
template <typename T> struct DBuf {
  T *p = nullptr;
  size_t cap = 0;
  int ensure(size_t n, cudaStream_t s) {
    if (n <= cap) return HZ_OK;
    size_t want = std::max(n, cap + cap / 2);
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
    if (n <= cap) return HZ_OK;
    size_t want = std::max(n, cap + cap / 2);
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
  return HZ_OK;
}

// --- dedup_and_order (src/hsp.rs:62-126) --------------------------------------
inline uint32_t diag_of(const hz_segment_pair &h) { return h.ref_start - h.query_start; }
bool by_diagonal(const hz_segment_pair &x, const hz_segment_pair &y) {
  uint32_t dx = diag_of(x), dy = diag_of(y);
  if (dx != dy) return dx < dy;
  if (x.ref_start != y.ref_start) return x.ref_start < y.ref_start;
  if (x.len != y.len) return x.len < y.len;
  return x.score > y.score;
}
bool by_lastz(const hz_segment_pair &x, const hz_segment_pair &y) {
  if (x.query_start != y.query_start) return x.query_start < y.query_start;
  if (x.ref_start != y.ref_start) return x.ref_start < y.ref_start;
  if (x.len != y.len) return x.len < y.len;
  return x.score > y.score;
}
bool contained(const hz_segment_pair &x, const hz_segment_pair &y) {
  uint32_t xe = x.ref_start + x.len, ye = y.ref_start + y.len;
  return diag_of(x) == diag_of(y) &&
         ((x.ref_start >= y.ref_start && xe <= ye) || (y.ref_start >= x.ref_start && ye <= xe));
}
// Both orders are total over the four fields, so std::sort reproduces the
// reference's stable sorts exactly.
size_t dedup_and_order(hz_segment_pair *h, size_t n) {
  if (n == 0) return 0;
  std::sort(h, h + n, by_diagonal);
  size_t k = 1;
  hz_segment_pair prev = h[0];
  for (size_t i = 1; i < n; i++) {
    hz_segment_pair cur = h[i];
    if (!contained(prev, cur)) h[k++] = cur;
    prev = cur;
  }
  std::sort(h, h + k, by_lastz);
  return k;
}

unsigned grid_for(uint64_t n, unsigned threads, unsigned cap = 148u * 64u) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return (unsigned)std::min<uint64_t>(b, cap);
}

}  // namespace

// ---------------------------------------------------------------------------

struct Slot {
  int kind = 0;  // 0 empty, 1 uploaded seeds, 2 generated on device
  DBuf<uint64_t> seeds;
  uint64_t n_slots = 0;  // seed slots of the call (uploaded: seeds; generated: span * per_pos)
  uint64_t n_seeds = 0;  // real seeds (chunk_seeds count)
  int rev = 0;
  uint32_t start = 0, end = 0, per_pos = 1;
  DBuf<uint32_t> cnt, bst;
  bool counted = false;
};

struct ProfEntry {
  double ms = 0;
  uint64_t n = 0;
};

struct hz_engine {
  int device = 0;
  cudaStream_t st = nullptr;
  cudaStream_t own_st = nullptr;
  hz_config cfg;
  ShapeDev shape;
  ExtendParams ep;
  uint32_t max_hits = 0;
  // target
  DBuf<uint8_t> ref;
  uint32_t rlen = 0;
  DBuf<uint32_t> index_table;
  uint64_t index_len = 0;
  DBuf<uint32_t> pos_table;
  uint64_t n_pos = 0;
  bool has_target = false;
  // query
  DBuf<uint8_t> qf, qr, qascii;
  uint32_t qlen = 0;
  bool has_query = false;
  Slot slot[2];
  // per-call work
  DBuf<uint2> pairs, pair_partial, pair_total;
  DBuf<uint32_t> c_incl, c_qpos, c_bst, bounds, status, raw_count, bad;
  DBuf<uint64_t> anchors;
  DBuf<SegmentPair> raw;
  DBuf<unsigned long long> cells, n_valid;
  HBuf<uint8_t> h_stage;
  HBuf<hz_segment_pair> h_raw;
  HBuf<uint32_t> h_small;
  // profiling
  bool profiling = false;
  std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  std::vector<cudaEvent_t> event_pool;
  std::map<std::string, ProfEntry> prof;
  std::vector<std::string> prof_order;
  uint64_t launches = 0;

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
  // Brackets one launch with events when profiling.
  template <typename F> int launch(const char *name, F &&f) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (profiling) {
      a = get_event();
      b = get_event();
      cudaEventRecord(a, st);
    }
    f();
    launches++;
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return fail(HZ_E_CUDA, "launch %s: %s", name, cudaGetErrorString(err));
    if (profiling) {
      cudaEventRecord(b, st);
      pending.push_back({name, {a, b}});
    }
    return HZ_OK;
  }
  // Waits for the stream and folds finished event pairs into the profile.
  int sync() {
    CK(cudaStreamSynchronize(st));
    for (auto &pe : pending) {
      float ms = 0;
      cudaEventElapsedTime(&ms, pe.second.first, pe.second.second);
      if (!prof.count(pe.first)) prof_order.push_back(pe.first);
      prof[pe.first].ms += ms;
      prof[pe.first].n += 1;
      event_pool.push_back(pe.second.first);
      event_pool.push_back(pe.second.second);
    }
    pending.clear();
    return HZ_OK;
  }
};

namespace {

int set_device(hz_engine *e) {
  CK(cudaSetDevice(e->device));
  return HZ_OK;
}

// Exclusive scan of the (hits, non-empty) pairs of n seed slots; totals to
// host: *num_hits and *n_entries.
int scan_pairs(hz_engine *e, const uint32_t *cnt, uint64_t n, uint64_t *num_hits, uint64_t *n_entries) {
  TRY(e->pairs.ensure(n, e->st));
  TRY(e->pair_partial.ensure(scan_tiles(n) + 1, e->st));
  TRY(e->pair_total.ensure(1, e->st));
  uint2 *pairs = e->pairs.p;
  TRY(e->launch("pair", [&] { pair_kernel<<<grid_for(n, 256), 256, 0, e->st>>>(cnt, n, pairs); }));
  TRY(e->launch("scan", [&] {
    exclusive_scan<uint2>(pairs, pairs, n, e->pair_partial.p, e->pair_total.p, e->st);
  }));
  e->launches += 2;
  TRY(e->h_small.ensure(4));
  CK(cudaMemcpyAsync(e->h_small.p, e->pair_total.p, sizeof(uint2), cudaMemcpyDeviceToHost, e->st));
  TRY(e->sync());
  *num_hits = e->h_small.p[0];
  *n_entries = e->h_small.p[1];
  return HZ_OK;
}

// Everything after the seed lookup of one call: compaction, MAX_HITS walk,
// per-chunk expansion + extension, per-chunk dedup.  Appends to `out`.
int filter_slot(hz_engine *e, Slot &s, const uint8_t *qry, std::vector<hz_segment_pair> &out, hz_stats *st) {
  uint64_t n = s.n_slots;
  if (n == 0) return HZ_OK;
  uint64_t num_hits64 = 0, n_entries = 0;
  TRY(scan_pairs(e, s.cnt.p, n, &num_hits64, &n_entries));
  if (st) {
    st->hits += num_hits64;
    st->seeds += s.n_seeds;
    st->calls += 1;
  }
  if (num_hits64 == 0) return HZ_OK;
  if (num_hits64 > 0xFFFFFFFFull)
    return fail(HZ_E_INVALID, "a call holds %llu seed hits; num_hits is a u32 in the reference",
                (unsigned long long)num_hits64);
  uint32_t num_hits = (uint32_t)num_hits64;

  TRY(e->c_incl.ensure(n_entries, e->st));
  TRY(e->c_qpos.ensure(n_entries, e->st));
  TRY(e->c_bst.ensure(n_entries, e->st));
  const uint64_t *up = s.kind == 1 ? s.seeds.p : nullptr;
  TRY(e->launch("seed_compact", [&] {
    seed_compact_kernel<<<grid_for(n, 256), 256, 0, e->st>>>(s.cnt.p, s.bst.p, e->pairs.p, n, s.per_pos, s.start,
                                                              up, e->c_incl.p, e->c_qpos.p, e->c_bst.p);
  }));

  // chunk bounds in hit space
  std::vector<uint32_t> bounds;
  if (num_hits <= e->max_hits) {
    bounds = {0u, num_hits};
  } else {
    uint32_t num_iter = num_hits / e->max_hits + 1;
    TRY(e->bounds.ensure(num_iter + 1, e->st));
    TRY(e->status.ensure(1, e->st));
    // first real seed: the first slot with a bucket
    uint32_t first_hits = 0;
    {
      std::vector<uint32_t> hb;
      // scan forward on the host in blocks; this path only runs when a call
      // exceeds max_hits
      const uint64_t blk = 1 << 16;
      bool found = false;
      std::vector<uint32_t> c(blk), b(blk);
      for (uint64_t off = 0; off < n && !found; off += blk) {
        uint64_t m = std::min<uint64_t>(blk, n - off);
        CK(cudaMemcpyAsync(c.data(), s.cnt.p + off, m * 4, cudaMemcpyDeviceToHost, e->st));
        CK(cudaMemcpyAsync(b.data(), s.bst.p + off, m * 4, cudaMemcpyDeviceToHost, e->st));
        TRY(e->sync());
        for (uint64_t i = 0; i < m; i++)
          if (b[i] != kNoBucket) {
            first_hits = c[i];
            found = true;
            break;
          }
      }
    }
    uint32_t *bp = e->bounds.p, *sp = e->status.p;
    TRY(e->launch("chunk_walk", [&] {
      chunk_walk_kernel<<<1, 32, 0, e->st>>>(e->c_incl.p, (uint32_t)n_entries, num_hits, e->max_hits, first_hits, bp,
                                             sp);
    }));
    bounds.resize(num_iter + 1);
    uint32_t status = 0;
    CK(cudaMemcpyAsync(bounds.data(), bp, (num_iter + 1) * 4, cudaMemcpyDeviceToHost, e->st));
    CK(cudaMemcpyAsync(&status, sp, 4, cudaMemcpyDeviceToHost, e->st));
    TRY(e->sync());
    if (status)
      return fail(HZ_E_INVALID, "the first seed of a call holds more than max_hits=%u hits; the reference's "
                                "MAX_HITS walk has no valid cut there", e->max_hits);
  }

  for (size_t c = 0; c + 1 < bounds.size(); c++) {
    uint32_t lo = bounds[c], hi = bounds[c + 1];
    if (hi <= lo) continue;
    uint32_t nh = hi - lo;
    TRY(e->anchors.ensure(nh, e->st));
    TRY(e->raw.ensure(nh, e->st));
    TRY(e->raw_count.ensure(1, e->st));
    CK(cudaMemsetAsync(e->raw_count.p, 0, 4, e->st));
    uint64_t *an = e->anchors.p;
    TRY(e->launch("expand", [&] {
      expand_kernel<<<(nh + kExpandTile - 1) / kExpandTile, kExpandThreads, 0, e->st>>>(
          e->c_incl.p, e->c_qpos.p, e->c_bst.p, (uint32_t)n_entries, e->pos_table.p, lo, hi, e->shape.size, an);
    }));
    ExtendParams ep = e->ep;
    ep.qlen = e->qlen;
    TRY(e->launch("extend", [&] {
      extend_kernel<<<grid_for(nh, kExtendThreads, 148u * 16u), kExtendThreads, 0, e->st>>>(
          e->ref.p, qry, an, nh, ep, e->raw.p, nh, e->raw_count.p, e->cells.p);
    }));
    uint32_t nraw = 0;
    CK(cudaMemcpyAsync(&nraw, e->raw_count.p, 4, cudaMemcpyDeviceToHost, e->st));
    TRY(e->sync());
    if (nraw == 0) continue;
    TRY(e->h_raw.ensure(nraw));
    CK(cudaMemcpyAsync(e->h_raw.p, e->raw.p, (size_t)nraw * sizeof(hz_segment_pair), cudaMemcpyDeviceToHost,
                       e->st));
    TRY(e->sync());
    size_t kept = dedup_and_order(e->h_raw.p, nraw);
    out.insert(out.end(), e->h_raw.p, e->h_raw.p + kept);
    if (st) {
      st->raw_hsps += nraw;
      st->hsps += kept;
    }
  }
  return HZ_OK;
}

// Device seed lookup for positions [start, end) of one strand into slot s.
int generate_into(hz_engine *e, Slot &s, int rev, uint32_t start, uint32_t end, int transitions) {
  s.kind = 2;
  s.rev = rev;
  s.start = start;
  s.end = end;
  s.per_pos = transitions ? 1 + e->shape.kmer_size : 1;
  uint32_t span = end > start ? end - start : 0;
  s.n_slots = (uint64_t)span * s.per_pos;
  s.counted = true;
  if (span == 0) return HZ_OK;
  TRY(s.cnt.ensure(s.n_slots, e->st));
  TRY(s.bst.ensure(s.n_slots, e->st));
  const uint8_t *q = rev ? e->qr.p : e->qf.p;
  TRY(e->launch("seed_count", [&] {
    seed_count_kernel<<<grid_for(span, 256), 256, 0, e->st>>>(q, start, span, s.per_pos, e->shape,
                                                              e->index_table.p, e->cfg.occ_cap, s.cnt.p, s.bst.p,
                                                              e->n_valid.p);
  }));
  return HZ_OK;
}

int check_range(hz_engine *e, uint32_t start, uint32_t end) {
  if (end < start) return fail(HZ_E_INVALID, "seed range [%u, %u) is reversed", start, end);
  if (end > start && (uint64_t)end + e->shape.size - 1 > e->qlen)
    return fail(HZ_E_INVALID, "seed range [%u, %u) exceeds query length %u", start, end, e->qlen);
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
  e->cfg = *cfg;
  e->cfg.seed[63] = 0;
  e->shape = sh;
  memcpy(e->ep.sub, cfg->sub_mat, sizeof(e->ep.sub));
  e->ep.xdrop = cfg->xdrop;
  e->ep.hspthresh = cfg->hspthresh;
  e->ep.noentropy = cfg->noentropy ? 1u : 0u;
  if (e->cfg.step == 0) e->cfg.step = 1;
  if (e->cfg.wga_chunk == 0) e->cfg.wga_chunk = 250000;
  if (e->cfg.interval == 0) e->cfg.interval = 10000000;
  if (e->cfg.strand == 0 || e->cfg.strand > 3) {
    delete e;
    return fail(HZ_E_INVALID, "strand must be 1 (plus), 2 (minus) or 3 (both)");
  }
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
  if (rc == HZ_OK) rc = e->cells.ensure(1, e->st);
  if (rc == HZ_OK) rc = e->n_valid.ensure(1, e->st);
  if (rc == HZ_OK && cudaMemsetAsync(e->cells.p, 0, 8, e->st) != cudaSuccess) rc = fail(HZ_E_CUDA, "memset");
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
  e->ref.release();
  e->index_table.release();
  e->pos_table.release();
  e->qf.release();
  e->qr.release();
  e->qascii.release();
  for (auto &s : e->slot) {
    s.seeds.release();
    s.cnt.release();
    s.bst.release();
  }
  e->pairs.release();
  e->pair_partial.release();
  e->pair_total.release();
  e->c_incl.release();
  e->c_qpos.release();
  e->c_bst.release();
  e->bounds.release();
  e->status.release();
  e->raw_count.release();
  e->bad.release();
  e->anchors.release();
  e->raw.release();
  e->cells.release();
  e->n_valid.release();
  e->h_stage.release();
  e->h_raw.release();
  e->h_small.release();
  for (auto &pe : e->pending) {
    cudaEventDestroy(pe.second.first);
    cudaEventDestroy(pe.second.second);
  }
  for (auto ev : e->event_pool) cudaEventDestroy(ev);
  if (e->own_st) cudaStreamDestroy(e->own_st);
  delete e;
}

int hz_engine_load_tables(hz_engine *e, const uint32_t *index_table, uint64_t index_len, const uint32_t *pos_table,
                          uint64_t pos_len, const uint8_t *ref_seq, uint64_t ref_len) {
  if (!e || !index_table || !ref_seq || (pos_len && !pos_table)) return fail(HZ_E_INVALID, "null argument");
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
  TRY(set_device(e));
  TRY(e->index_table.ensure(index_len, e->st));
  TRY(e->pos_table.ensure(pos_len + 1, e->st));
  TRY(e->ref.ensure(ref_len + 1, e->st));
  CK(cudaMemcpyAsync(e->index_table.p, index_table, index_len * 4, cudaMemcpyHostToDevice, e->st));
  if (pos_len) CK(cudaMemcpyAsync(e->pos_table.p, pos_table, pos_len * 4, cudaMemcpyHostToDevice, e->st));
  CK(cudaMemcpyAsync(e->ref.p, ref_seq, ref_len, cudaMemcpyHostToDevice, e->st));
  TRY(e->sync());
  e->index_len = index_len;
  e->n_pos = pos_len;
  e->rlen = (uint32_t)ref_len;
  e->ep.rlen = e->rlen;
  e->has_target = true;
  return HZ_OK;
}

int hz_engine_load_target(hz_engine *e, const uint8_t *ref_ascii, uint64_t len) {
  if (!e || (!ref_ascii && len)) return fail(HZ_E_INVALID, "null argument");
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
  DBuf<uint8_t> ascii, junk;
  TRY(ascii.ensure(len + 1, st));
  TRY(e->ref.ensure(len + 1, st));
  TRY(junk.ensure(len + 1, st));
  CK(cudaMemcpyAsync(ascii.p, ref_ascii, len, cudaMemcpyHostToDevice, st));
  if (len)
    TRY(e->launch("encode", [&] {
      encode_kernel<<<grid_for(len / 4 + 1, 256), 256, 0, st>>>(ascii.p, len, e->ref.p, junk.p);
    }));
  TRY(e->index_table.ensure(index_len, st));
  CK(cudaMemsetAsync(e->index_table.p, 0, index_len * 4, st));

  DBuf<uint32_t> kmers, flags, keys, vals, keys2, vals2, partial, total, hist, hpartial;
  uint64_t n_valid = 0;
  if (num_steps) {
    TRY(kmers.ensure(num_steps, st));
    TRY(flags.ensure(num_steps, st));
    TRY(partial.ensure(scan_tiles(num_steps) + 1, st));
    TRY(total.ensure(1, st));
    TRY(e->launch("ref_kmer", [&] {
      ref_kmer_kernel<<<grid_for(num_steps, 256), 256, 0, st>>>(e->ref.p, num_steps, start_offset, step, sh, kmers.p,
                                                                flags.p);
    }));
    TRY(e->launch("ref_scan", [&] { exclusive_scan<uint32_t>(flags.p, flags.p, num_steps, partial.p, total.p, st); }));
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
    kmers.release();
    flags.release();
    // stable radix sort by k-mer, 8 bits per pass
    if (n_valid) {
      TRY(keys2.ensure(n_valid + 1, st));
      TRY(vals2.ensure(n_valid + 1, st));
      uint64_t tiles = (n_valid + kRadixTile - 1) / kRadixTile;
      TRY(hist.ensure(tiles * kRadixBins, st));
      TRY(hpartial.ensure(scan_tiles(tiles * kRadixBins) + 1, st));
      int bits = 2 * (int)sh.kmer_size;
      uint32_t *ka = keys.p, *va = vals.p, *kb = keys2.p, *vb = vals2.p;
      for (int shift = 0; shift < bits; shift += 8) {
        TRY(e->launch("radix_hist", [&] {
          radix_hist_kernel<<<(unsigned)tiles, kRadixThreads, 0, st>>>(ka, n_valid, shift, hist.p, tiles);
        }));
        TRY(e->launch("radix_scan", [&] {
          exclusive_scan<uint32_t>(hist.p, hist.p, tiles * kRadixBins, hpartial.p, total.p, st);
        }));
        TRY(e->launch("radix_scatter", [&] {
          radix_scatter_kernel<<<(unsigned)tiles, kRadixThreads, 0, st>>>(ka, va, n_valid, shift, hist.p, tiles, kb,
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
  // index_table = inclusive cumulative bucket counts
  {
    DBuf<uint32_t> excl, ipart;
    TRY(excl.ensure(index_len, st));
    TRY(ipart.ensure(scan_tiles(index_len) + 1, st));
    TRY(total.ensure(1, st));
    TRY(e->launch("index_scan", [&] {
      exclusive_scan<uint32_t>(e->index_table.p, excl.p, index_len, ipart.p, total.p, st);
    }));
    TRY(e->launch("index_add", [&] {
      add_counts_kernel<<<grid_for(index_len, 256), 256, 0, st>>>(excl.p, e->index_table.p, index_len);
    }));
    CK(cudaMemcpyAsync(e->index_table.p, excl.p, index_len * 4, cudaMemcpyDeviceToDevice, st));
    TRY(e->sync());
    excl.release();
    ipart.release();
  }
  ascii.release();
  junk.release();
  keys.release();
  vals.release();
  keys2.release();
  vals2.release();
  partial.release();
  total.release();
  hist.release();
  hpartial.release();
  e->index_len = index_len;
  e->n_pos = n_valid;
  e->rlen = (uint32_t)len;
  e->ep.rlen = e->rlen;
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
  TRY(set_device(e));
  TRY(e->qf.ensure(len + 1, e->st));
  TRY(e->qr.ensure(len + 1, e->st));
  CK(cudaMemcpyAsync(e->qf.p, query, len, cudaMemcpyHostToDevice, e->st));
  CK(cudaMemcpyAsync(e->qr.p, query_rc, len, cudaMemcpyHostToDevice, e->st));
  TRY(e->sync());
  e->qlen = (uint32_t)len;
  e->has_query = true;
  e->slot[0].kind = e->slot[1].kind = 0;
  return HZ_OK;
}

int hz_swap_query_ascii(hz_engine *e, const uint8_t *q, uint64_t len) {
  if (!e || (len && !q)) return fail(HZ_E_INVALID, "null argument");
  if (len > 0xFFFFFFFFull) return fail(HZ_E_INVALID, "query block exceeds u32 coordinates");
  TRY(set_device(e));
  TRY(e->qascii.ensure(len + 1, e->st));
  TRY(e->qf.ensure(len + 1, e->st));
  TRY(e->qr.ensure(len + 1, e->st));
  CK(cudaMemcpyAsync(e->qascii.p, q, len, cudaMemcpyHostToDevice, e->st));
  if (len)
    TRY(e->launch("encode", [&] {
      encode_kernel<<<grid_for(len / 4 + 1, 256), 256, 0, e->st>>>(e->qascii.p, len, e->qf.p, e->qr.p);
    }));
  TRY(e->sync());
  e->qlen = (uint32_t)len;
  e->has_query = true;
  e->slot[0].kind = e->slot[1].kind = 0;
  return HZ_OK;
}

int hz_upload_seeds(hz_engine *e, uint32_t slot, const uint64_t *seeds, uint64_t n) {
  if (!e || slot > 1 || (n && !seeds)) return fail(HZ_E_INVALID, "bad argument");
  TRY(set_device(e));
  Slot &s = e->slot[slot];
  TRY(s.seeds.ensure(n + 1, e->st));
  if (n) CK(cudaMemcpyAsync(s.seeds.p, seeds, n * 8, cudaMemcpyHostToDevice, e->st));
  TRY(e->sync());
  s.kind = 1;
  s.n_slots = n;
  s.n_seeds = n;
  s.per_pos = 1;
  s.start = 0;
  s.counted = false;
  return HZ_OK;
}

int hz_generate_seeds(hz_engine *e, uint32_t slot, int rev, uint32_t start, uint32_t end, int transitions,
                      uint64_t *n_seeds) {
  if (!e || slot > 1) return fail(HZ_E_INVALID, "bad argument");
  if (!e->has_query) return fail(HZ_E_STATE, "Engine has no query: swap_query() must be called before generate_seeds()");
  if (!e->has_target) return fail(HZ_E_STATE, "no target loaded");
  TRY(check_range(e, start, end));
  TRY(set_device(e));
  CK(cudaMemsetAsync(e->n_valid.p, 0, 8, e->st));
  TRY(generate_into(e, e->slot[slot], rev, start, end, transitions));
  unsigned long long nv = 0;
  CK(cudaMemcpyAsync(&nv, e->n_valid.p, 8, cudaMemcpyDeviceToHost, e->st));
  TRY(e->sync());
  e->slot[slot].n_seeds = nv * e->slot[slot].per_pos;
  if (n_seeds) *n_seeds = e->slot[slot].n_seeds;
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
  if (s.kind == 2 && s.rev != rev) return fail(HZ_E_INVALID, "slot %u was generated for the other strand", slot);
  hz_stats local;
  memset(&local, 0, sizeof local);
  const uint8_t *q = rev ? e->qr.p : e->qf.p;
  if (s.kind == 1 && !s.counted) {
    TRY(s.cnt.ensure(s.n_slots + 1, e->st));
    TRY(s.bst.ensure(s.n_slots + 1, e->st));
    TRY(e->bad.ensure(1, e->st));
    CK(cudaMemsetAsync(e->bad.p, 0, 4, e->st));
    uint32_t max_pos = e->qlen >= e->shape.size ? e->qlen - e->shape.size : 0;
    if (s.n_slots) {
      uint64_t ns = s.n_slots;
      TRY(e->launch("seed_count", [&] {
        seed_count_uploaded_kernel<<<grid_for(ns, 256), 256, 0, e->st>>>(s.seeds.p, ns, e->index_table.p,
                                                                         e->cfg.occ_cap, (uint32_t)e->index_len, max_pos,
                                                                         s.cnt.p, s.bst.p, e->bad.p);
      }));
    }
    uint32_t bad = 0;
    CK(cudaMemcpyAsync(&bad, e->bad.p, 4, cudaMemcpyDeviceToHost, e->st));
    TRY(e->sync());
    if (bad) return fail(HZ_E_INVALID, "an uploaded seed has a k-mer or position outside the tables/query");
    s.counted = true;
  }
  CK(cudaMemsetAsync(e->cells.p, 0, 8, e->st));
  std::vector<hz_segment_pair> res;
  TRY(filter_slot(e, s, q, res, &local));
  unsigned long long cells = 0;
  CK(cudaMemcpyAsync(&cells, e->cells.p, 8, cudaMemcpyDeviceToHost, e->st));
  TRY(e->sync());
  local.cells = cells;
  if (!res.empty()) {
    *out = (hz_segment_pair *)malloc(res.size() * sizeof(hz_segment_pair));
    if (!*out) return fail(HZ_E_OOM, "host allocation");
    memcpy(*out, res.data(), res.size() * sizeof(hz_segment_pair));
  }
  *n = res.size();
  if (stats) *stats = local;
  return HZ_OK;
}

int hz_run_pass(hz_engine *e, hz_pass_record **out, uint64_t *n, hz_stats *stats) {
  if (!e || !out || !n) return fail(HZ_E_INVALID, "bad argument");
  *out = nullptr;
  *n = 0;
  if (!e->has_query) return fail(HZ_E_STATE, "Engine has no query: swap_query() must be called first");
  if (!e->has_target) return fail(HZ_E_STATE, "no target loaded");
  TRY(set_device(e));
  hz_stats local;
  memset(&local, 0, sizeof local);
  uint32_t ss = e->shape.size;
  uint64_t qlen = e->qlen;
  // intervals (src/sequence.rs:322-334) and the batch list (src/run.rs:278-299)
  std::vector<std::pair<uint32_t, uint32_t>> iv;
  if (qlen > ss) {
    uint32_t end_pos = (uint32_t)(qlen - ss);
    for (uint64_t cur = 0; cur < end_pos; cur += e->cfg.interval)
      iv.push_back({(uint32_t)cur, (uint32_t)std::min<uint64_t>(end_pos, cur + e->cfg.interval)});
  }
  uint32_t qbl = qlen > ss ? (uint32_t)(qlen - ss) : 0;
  std::vector<hz_pass_record> recs;
  CK(cudaMemsetAsync(e->cells.p, 0, 8, e->st));
  CK(cudaMemsetAsync(e->n_valid.p, 0, 8, e->st));
  Slot &s = e->slot[0];
  for (size_t i = 0; i < iv.size(); i++) {
    std::vector<hz_segment_pair> per[2];
    for (int rev = 0; rev < 2; rev++) {
      if (!(e->cfg.strand & (1u << rev))) continue;
      uint32_t a = rev ? qbl - iv[i].second : iv[i].first;
      uint32_t b = rev ? qbl - iv[i].first : iv[i].second;
      for (uint64_t c = a; c < b; c += e->cfg.wga_chunk) {  // chunks(), src/seed.rs:488-496
        uint32_t cs = (uint32_t)c, ce = (uint32_t)std::min<uint64_t>(c + e->cfg.wga_chunk, (uint64_t)b + 1);
        TRY(generate_into(e, s, rev, cs, ce, e->cfg.transitions));
        s.n_seeds = 0;
        TRY(filter_slot(e, s, rev ? e->qr.p : e->qf.p, per[rev], &local));
      }
    }
    for (int rev = 0; rev < 2; rev++)
      for (auto &h : per[rev]) recs.push_back({(uint32_t)i, (uint32_t)rev, h});
  }
  unsigned long long cells = 0, nv = 0;
  CK(cudaMemcpyAsync(&cells, e->cells.p, 8, cudaMemcpyDeviceToHost, e->st));
  CK(cudaMemcpyAsync(&nv, e->n_valid.p, 8, cudaMemcpyDeviceToHost, e->st));
  TRY(e->sync());
  local.cells = cells;
  local.seeds = nv * (e->cfg.transitions ? 1 + e->shape.kmer_size : 1);
  // calls with no seeds are not calls in the reference (src/run.rs:431)
  if (!recs.empty()) {
    *out = (hz_pass_record *)malloc(recs.size() * sizeof(hz_pass_record));
    if (!*out) return fail(HZ_E_OOM, "host allocation");
    memcpy(*out, recs.data(), recs.size() * sizeof(hz_pass_record));
  }
  *n = recs.size();
  if (stats) *stats = local;
  e->slot[0].kind = 0;
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

uint64_t hz_engine_launches(hz_engine *e) { return e ? e->launches : 0; }

int hz_engine_set_stream(hz_engine *e, void *stream) {
  if (!e) return fail(HZ_E_INVALID, "null engine");
  TRY(set_device(e));
  TRY(e->sync());
  e->st = stream ? (cudaStream_t)stream : e->own_st;
  return HZ_OK;
}

}  // extern "C"
