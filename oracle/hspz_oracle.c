/*
 * hspz_oracle.c -- CPU restatement of hspZ's seed-and-filter path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle and the timed
 * CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs
 * load it, and only as the checker.  The product (hspz_b200) never links,
 * loads or calls it.
 *
 * Parity pin: the fixtures of assets/tests/gen_fixtures.py, run through this
 * oracle and rendered as .segments, reproduce the reference's frozen smoke
 * digests (assets/container/smoke.sh:11-12: repeat 57 HSPs d01edd2118cf5fa5,
 * multi 3 HSPs 0da3bbda656e4f7b) -- see tests/test_oracle_golden.py.
 *
 * Every function cites the reference file:line it restates.  Integer work is
 * done in uint32 arithmetic where the reference wraps (Rust release builds and
 * the GPU wrap on i32 overflow), so that no C signed-overflow UB is involved.
 * The only floating-point step (entropy, src/gpu/kernels.rs:1555-1701) is a
 * fixed sequence of IEEE double operations with no FMA contraction; build with
 * -ffp-contract=off.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define HZO_INVALID_KMER (1u << 31) /* src/seed.rs:27 */
#define HZO_NUC 8                   /* src/sequence.rs:43 */

/* ------------------------------------------------------------------------ */
/* Alphabet (src/sequence.rs:35-86)                                          */

/* encode(): ASCII -> device alphabet.  src/sequence.rs:66-79 */
static uint8_t enc_of(uint8_t c) {
  switch (c) {
    case 'A': return 0;
    case 'C': return 1;
    case 'G': return 2;
    case 'T': return 3;
    case 'a': case 'c': case 'g': case 't': return 4; /* L_NT */
    case 'n': case 'N': return 5;                      /* N_NT */
    case '&': return 7;                                /* E_NT */
    default: return 6;                                 /* X_NT */
  }
}

void hzo_encode(const uint8_t *s, uint64_t n, uint8_t *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = enc_of(s[i]);
}

/* REV_COMP table, src/sequence.rs:83-86 (IUPAC-aware, >=128 -> 'N'). */
static const char REV_COMP[129] =
    "NNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNN"
    "NNNNNN&NNNNNNNNNNNNNNNNNNNNNNNNN"
    "NTVGHNNCDNNMNKNNNNYSAABWNRNNNNNN"
    "NtvghnncdnnmnknnnnysaabwnrnNNNNN";

/* reverse_complement() of a block.  src/sequence.rs:212-230 */
void hzo_revcomp(const uint8_t *s, uint64_t n, uint8_t *out) {
  for (uint64_t i = 0; i < n; i++) {
    uint8_t c = s[n - 1 - i];
    out[i] = c < 128 ? (uint8_t)REV_COMP[c] : (uint8_t)'N';
  }
}

/* ------------------------------------------------------------------------ */
/* Shape (src/seed.rs:34-123)                                                */

typedef struct {
  uint32_t size;       /* pattern width */
  uint32_t kmer_size;  /* care positions */
  uint32_t pos[32];
  uint32_t transition[32];
} hzo_shape;

/* Shape::parse.  src/seed.rs:49-79 */
int hzo_shape_parse(const char *spec, hzo_shape *out) {
  const char *pat = spec;
  if (strcmp(spec, "12of19") == 0) pat = "TTT0T00TT00T0T0TTTT";
  else if (strcmp(spec, "14of22") == 0) pat = "TTT0T0TT00TT00T0T0TTTT";
  memset(out, 0, sizeof(*out));
  uint32_t n = 0, k = 0;
  for (const char *c = pat; *c; c++, n++) {
    /* custom patterns: '1' and 'T' both become 'T' (all transition-allowed) */
    if (*c == '1' || *c == 'T') {
      if (k >= 32) return -1;
      out->pos[k] = n;
      out->transition[k] = 1;
      k++;
    }
  }
  if (k < 4 || k > 15) return -1;
  out->size = n;
  out->kmer_size = k;
  return 0;
}

/* Shape::kmer_at on device codes (code < 4 <=> uppercase ACGT, the seeding
 * alphabet of nt_char_to_int).  The WHOLE window must be codeable.
 * src/seed.rs:88-101 */
static inline uint32_t kmer_at(const uint8_t *codes, uint64_t pos, const hzo_shape *sh) {
  for (uint32_t i = 0; i < sh->size; i++)
    if (codes[pos + i] >= 4) return HZO_INVALID_KMER;
  uint32_t kmer = 0;
  for (uint32_t t = 0; t < sh->kmer_size; t++) kmer = (kmer << 2) + codes[pos + sh->pos[t]];
  return kmer;
}

/* ------------------------------------------------------------------------ */
/* Seed table (src/seed.rs:135-180, hit_count :365-373)                      */

/* SeedTable::build.  index_table has 4^kmer_size entries (inclusive
 * cumulative counts); pos_table is malloc'd here, buckets in ascending
 * position order.  At step 1 position 0 is never indexed (start_offset 1). */
int hzo_seed_table_build(const uint8_t *codes, uint64_t len, const hzo_shape *sh,
                         uint32_t step, uint32_t *index_table, uint32_t **pos_table,
                         uint64_t *n_pos) {
  if (step < 1) step = 1;
  uint64_t offset = (sh->size + 1) % step;
  uint64_t start_offset = step - offset;
  uint64_t table = 1ull << (2 * sh->kmer_size);
  uint64_t num_steps = (len + offset) > sh->size ? (len + offset - sh->size) / step : 0;
  uint64_t *counts = calloc(table + 1, sizeof(uint64_t));
  uint32_t *idxs = malloc((num_steps ? num_steps : 1) * sizeof(uint32_t));
  if (!counts || !idxs) { free(counts); free(idxs); return -1; }
  for (uint64_t i = 0; i < num_steps; i++) {
    uint32_t k = kmer_at(codes, start_offset + i * step, sh);
    idxs[i] = k;
    if (k != HZO_INVALID_KMER) counts[k + 1]++;
  }
  for (uint64_t i = 1; i <= table; i++) counts[i] += counts[i - 1];
  uint64_t total = counts[table];
  uint32_t *pt = malloc((total ? total : 1) * sizeof(uint32_t));
  if (!pt) { free(counts); free(idxs); return -1; }
  for (uint64_t i = 0; i < num_steps; i++) {
    uint32_t k = idxs[i];
    if (k != HZO_INVALID_KMER) pt[counts[k]++] = (uint32_t)(start_offset + i * step);
  }
  /* counts[k] now holds the inclusive end of bucket k == index_table[k] */
  for (uint64_t k = 0; k < table; k++) index_table[k] = (uint32_t)counts[k];
  free(counts);
  free(idxs);
  *pos_table = pt;
  *n_pos = total;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Parameters and records                                                    */

typedef struct {
  int32_t sub_mat[64];   /* build_sub_mat, src/scoring.rs:41-120 */
  int32_t xdrop;
  int32_t hspthresh;
  uint32_t noentropy;
  uint32_t max_hits;     /* pinned; must be > 0 */
  uint32_t occ_cap;      /* per-seed occurrence cap; 0 = none (build extension) */
  uint32_t transitions;
  uint32_t wga_chunk;    /* -C, default 250000 */
  uint32_t interval;     /* -I, default 10000000 */
  uint32_t strand;       /* bit0 plus, bit1 minus */
  uint32_t threads;
} hzo_params;

typedef struct {
  uint32_t ref_start, query_start, len;
  int32_t score;
} hzo_hsp; /* SegmentPair, src/hsp.rs:31-41 */

typedef struct {
  uint64_t seeds, hits, raw_hsps, hsps, cells, calls;
} hzo_stats;

enum { HZO_OK = 0, HZO_E_INVALID = -22, HZO_E_OOM = -12 };

/* ------------------------------------------------------------------------ */
/* hspZ's own natural log: an atanh series over the reduced mantissa,        */
/* src/gpu/kernels.rs:1879-1908.  Restated operation for operation so the    */
/* entropy is bit-identical between this oracle and the CUDA kernel.          */

static const double HZO_LN2 = 0x1.62e42fefa39efp-1;   /* f64 LN_2 */
static const double HZO_SQRT2 = 0x1.6a09e667f3bcdp+0; /* f64 SQRT_2 */
static const double HZO_LOG4 = 1.3862943649291992;     /* (double)logf(4.0f), src/gpu/mod.rs:2349-2352 */

static double hzo_ln(double x) {
  uint64_t bits;
  memcpy(&bits, &x, 8);
  int32_t ex = (int32_t)((bits >> 52) & 0x7FF) - 1023;
  uint64_t mb = (bits & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
  double m;
  memcpy(&m, &mb, 8);
  if (m > HZO_SQRT2) {
    m = m * 0.5;
    ex += 1;
  }
  double s = (m - 1.0) / (m + 1.0);
  double z = s * s;
  double poly = 1.0 + z * (1.0 / 3.0 + z * (1.0 / 5.0 + z * (1.0 / 7.0 + z * (1.0 / 9.0 +
                z * (1.0 / 11.0 + z * (1.0 / 13.0 + z * (1.0 / 15.0)))))));
  return 2.0 * s * poly + (double)ex * HZO_LN2;
}

double hzo_ln_export(double x) { return hzo_ln(x); }

/* Rust `f64 as i32`: truncation toward zero, saturating, NaN -> 0. */
static int32_t sat_i32(double v) {
  if (v != v) return 0;
  if (v >= 2147483647.0) return 2147483647;
  if (v <= -2147483648.0) return (int32_t)0x80000000u;
  return (int32_t)v;
}

/* ------------------------------------------------------------------------ */
/* Ungapped X-drop extension of one seed hit, scalar form of find_hsps       */
/* (src/gpu/kernels.rs:1279-1406 right, :1417-1543 left, entropy and accept  */
/* :1555-1701).                                                              */
/*                                                                          */
/* Anchor (r, q) is the END of the seed window (pos + seed_size,            */
/* src/gpu/kernels.rs:397-401).  Right cells are (r+k, q+k); left cells are */
/* (r-1-k, q-1-k).  Per cell: S += sub; the running maximum M' = max(M, S)  */
/* includes the cell; the extension stops at the first cell with            */
/* M' - S > xdrop, and the returned maximum is the one BEFORE that cell     */
/* (the warp kernel reads lane first-1).  Ties keep the earliest position.  */
/* Right position starts at -1 (offset of the max cell), left at 0 (count   */
/* of bases).                                                               */

typedef struct {
  int32_t accepted;
  hzo_hsp hsp;
  uint64_t cells;
  int32_t total;
} hzo_ext;

static hzo_ext extend_hit(const uint8_t *ref, uint32_t rlen, const uint8_t *qry, uint32_t qlen,
                          const hzo_params *p, uint32_t r, uint32_t q) {
  const int32_t *sub = p->sub_mat;
  hzo_ext out;
  memset(&out, 0, sizeof(out));
  uint64_t cells = 0;

  /* right */
  int32_t S = 0, M = 0, rpos = -1;
  for (uint32_t k = 0;; k++) {
    uint32_t rp = r + k, qp = q + k;
    if (!(rp < rlen && qp < qlen)) break;
    cells++;
    S = (int32_t)((uint32_t)S + (uint32_t)sub[ref[rp] * HZO_NUC + qry[qp]]);
    int32_t Mn = S > M ? S : M;
    if ((int32_t)((uint32_t)Mn - (uint32_t)S) > p->xdrop) break;
    if (S > M) { M = S; rpos = (int32_t)k; }
  }
  int32_t rmax = M;

  /* left */
  S = 0; M = 0;
  int32_t lpos = 0;
  for (uint32_t k = 0;; k++) {
    if (!(r >= k + 1 && q >= k + 1)) break;
    uint32_t rp = r - 1 - k, qp = q - 1 - k;
    cells++;
    S = (int32_t)((uint32_t)S + (uint32_t)sub[ref[rp] * HZO_NUC + qry[qp]]);
    int32_t Mn = S > M ? S : M;
    if ((int32_t)((uint32_t)Mn - (uint32_t)S) > p->xdrop) break;
    if (S > M) { M = S; lpos = (int32_t)(k + 1); }
  }
  int32_t lmax = M;

  int32_t total = (int32_t)((uint32_t)rmax + (uint32_t)lmax);
  int32_t extent = (int32_t)((uint32_t)rpos + (uint32_t)lpos);
  double entropy = 1.0;
  int32_t T = p->hspthresh;
  int32_t T3 = (int32_t)((uint32_t)T * 3u);
  if (total >= T && total <= T3 && p->noentropy == 0) {
    uint32_t rs = r - (uint32_t)lpos, qs = q - (uint32_t)lpos;
    int32_t positions = (int32_t)((uint32_t)extent + 1u);
    /* four 16-bit counters packed in one u64, as the kernel accumulates them */
    uint64_t packed = 0;
    for (int32_t i = 0; i < positions; i++) {
      uint8_t a = ref[rs + (uint32_t)i], b = qry[qs + (uint32_t)i];
      if (a == b && a < 4) packed += 1ull << (16 * a);
    }
    int32_t count[4] = {(int32_t)(packed & 0xFFFF), (int32_t)((packed >> 16) & 0xFFFF),
                        (int32_t)((packed >> 32) & 0xFFFF), (int32_t)((packed >> 48) & 0xFFFF)};
    int32_t total_count = count[0] + count[1] + count[2] + count[3];
    if (total_count >= 20) {
      double denom = (double)((int32_t)((uint32_t)extent + 1u));
      double ent = 0.0;
      for (int i = 0; i < 4; i++) {
        double pr = (double)count[i] / denom;
        double lg = count[i] != 0 ? hzo_ln(pr) : 0.0;
        ent = ent + pr * lg;
      }
      entropy = -ent / HZO_LOG4;
    }
  }
  out.cells = cells;
  out.total = total;
  double upper = (double)(float)total;
  if (sat_i32(upper * entropy) >= T) {
    out.accepted = 1;
    out.hsp.ref_start = r - (uint32_t)lpos;
    out.hsp.query_start = q - (uint32_t)lpos;
    out.hsp.len = (uint32_t)extent;
    out.hsp.score = entropy > 0.0 ? sat_i32((double)total * entropy) : 0;
  }
  return out;
}

/* exported for unit tests of single extensions */
int hzo_extend_hit(const uint8_t *ref, uint32_t rlen, const uint8_t *qry, uint32_t qlen,
                   const hzo_params *p, uint32_t r, uint32_t q, hzo_hsp *hsp, uint64_t *cells,
                   int32_t *total) {
  hzo_ext e = extend_hit(ref, rlen, qry, qlen, p, r, q);
  *hsp = e.hsp;
  *cells = e.cells;
  *total = e.total;
  return e.accepted;
}

/* ------------------------------------------------------------------------ */
/* Dedup (src/hsp.rs:49-126)                                                 */

static inline uint32_t diag_of(const hzo_hsp *h) { return h->ref_start - h->query_start; }

/* hspComp: diagonal, ref_start, len ascending, score descending. */
static int by_diagonal(const void *a, const void *b) {
  const hzo_hsp *x = a, *y = b;
  uint32_t dx = diag_of(x), dy = diag_of(y);
  if (dx != dy) return dx < dy ? -1 : 1;
  if (x->ref_start != y->ref_start) return x->ref_start < y->ref_start ? -1 : 1;
  if (x->len != y->len) return x->len < y->len ? -1 : 1;
  if (x->score != y->score) return x->score > y->score ? -1 : 1;
  return 0;
}

/* hspCompLastz: query_start, ref_start, len ascending, score descending. */
static int by_lastz(const void *a, const void *b) {
  const hzo_hsp *x = a, *y = b;
  if (x->query_start != y->query_start) return x->query_start < y->query_start ? -1 : 1;
  if (x->ref_start != y->ref_start) return x->ref_start < y->ref_start ? -1 : 1;
  if (x->len != y->len) return x->len < y->len ? -1 : 1;
  if (x->score != y->score) return x->score > y->score ? -1 : 1;
  return 0;
}

/* hspEqual: same diagonal and one ref interval [s, s+len] inside the other. */
static int contained(const hzo_hsp *x, const hzo_hsp *y) {
  uint32_t xe = x->ref_start + x->len, ye = y->ref_start + y->len;
  return diag_of(x) == diag_of(y) &&
         ((x->ref_start >= y->ref_start && xe <= ye) || (y->ref_start >= x->ref_start && ye <= xe));
}

/* dedup_and_order: sort by diagonal, keep i iff i == 0 or !contained(a[i-1],
 * a[i]) -- against the previous INPUT element -- then sort kept by lastz.
 * Both orders are total on all four fields, so an unstable sort gives the same
 * result as the reference's stable sort.  Returns the kept count (in place). */
uint64_t hzo_dedup_and_order(hzo_hsp *h, uint64_t n) {
  if (n == 0) return 0;
  qsort(h, n, sizeof(hzo_hsp), by_diagonal);
  uint64_t k = 1;
  hzo_hsp prev = h[0];
  for (uint64_t i = 1; i < n; i++) {
    hzo_hsp cur = h[i];
    if (!contained(&prev, &cur)) h[k++] = cur;
    prev = cur;
  }
  qsort(h, k, sizeof(hzo_hsp), by_lastz);
  return k;
}

/* ------------------------------------------------------------------------ */
/* One seed_and_filter call (src/gpu/mod.rs:1499-2178) with the MAX_HITS     */
/* chunk walk (chunk_limits, :2394-2420).                                    */

typedef struct {
  hzo_hsp *v;
  uint64_t n, cap;
} hsp_vec;

static int vec_push(hsp_vec *v, hzo_hsp h) {
  if (v->n == v->cap) {
    uint64_t nc = v->cap ? v->cap * 2 : 64;
    hzo_hsp *nv = realloc(v->v, nc * sizeof(hzo_hsp));
    if (!nv) return -1;
    v->v = nv;
    v->cap = nc;
  }
  v->v[v->n++] = h;
  return 0;
}

typedef struct {
  const hzo_params *p;
  const hzo_shape *sh;
  const uint8_t *ref;
  uint32_t rlen;
  const uint32_t *index_table;
  const uint32_t *pos_table;
} hzo_target;

/* Seeds of one WGA chunk in chunk_seeds order (src/seed.rs:385-398,
 * push_seeds :107-123): per valid position j ascending, the exact k-mer and
 * then, with transitions on, one variant per care position t (flip 2<<2t). */
static uint64_t gen_seeds(const hzo_shape *sh, const hzo_params *p, const uint8_t *qry,
                          uint32_t start, uint32_t end, uint64_t *seeds) {
  uint64_t n = 0;
  for (uint32_t j = start; j < end; j++) {
    uint32_t kmer = kmer_at(qry, j, sh);
    if (kmer == HZO_INVALID_KMER) continue;
    seeds[n++] = ((uint64_t)kmer << 32) | j;
    if (p->transitions)
      for (uint32_t t = 0; t < sh->kmer_size; t++)
        if (sh->transition[t])
          seeds[n++] = ((uint64_t)(kmer ^ (2u << (2 * t))) << 32) | j;
  }
  return n;
}

/* find_num_hits with the occurrence cap (a build extension: a bucket larger
 * than occ_cap contributes no hits). src/gpu/kernels.rs:70-115 */
static inline uint32_t hit_count(const hzo_target *t, uint32_t k) {
  uint32_t end = t->index_table[k];
  uint32_t c = k > 0 ? end - t->index_table[k - 1] : end;
  if (t->p->occ_cap && c > t->p->occ_cap) c = 0;
  return c;
}

/* Runs one call on `seeds`.  Output (deduped per MAX_HITS chunk, lastz order,
 * concatenated) is appended to *out.  Returns 0 or a negative code. */
/* chunk_limits (src/gpu/mod.rs:2394-2420, single-chunk shortcut :1693-1705):
 * the MAX_HITS split of one call over the inclusive running hit counts
 * hit_num[0..ns).  Each cut is the last seed whose running count is below the
 * running limit (partition_point(v < limit) - 1); the next limit is that
 * count plus max_hits.  A first seed alone above the limit has no valid cut
 * (the reference panics there): HZO_E_INVALID.  *out is malloc'd. */
static int chunk_limits(const uint32_t *hit_num, uint64_t ns, uint32_t max_hits, uint32_t (**out)[4],
                        uint32_t *n_out) {
  uint32_t num_hits = hit_num[ns - 1];
  uint32_t(*ch)[4];
  if (num_hits <= max_hits) {
    ch = malloc(sizeof(*ch));
    if (!ch) return HZO_E_OOM;
    ch[0][0] = 0; ch[0][1] = (uint32_t)(ns - 1); ch[0][2] = 0; ch[0][3] = num_hits;
    *out = ch;
    *n_out = 1;
    return 0;
  }
  uint32_t num_iter = num_hits / max_hits + 1;
  ch = malloc((uint64_t)num_iter * sizeof(*ch));
  if (!ch) return HZO_E_OOM;
  uint32_t limit = max_hits, start_seed = 0, start_hit = 0;
  for (uint32_t it = 0; it + 1 < num_iter; it++) {
    uint64_t lo = 0, hi = ns;
    while (lo < hi) {
      uint64_t mid = (lo + hi) / 2;
      if (hit_num[mid] < limit) lo = mid + 1; else hi = mid;
    }
    if (lo == 0) { free(ch); return HZO_E_INVALID; }
    uint32_t pos = (uint32_t)(lo - 1);
    ch[it][0] = start_seed; ch[it][1] = pos; ch[it][2] = start_hit; ch[it][3] = hit_num[pos];
    start_seed = pos + 1;
    start_hit = hit_num[pos];
    limit = hit_num[pos] + max_hits;
  }
  ch[num_iter - 1][0] = start_seed; ch[num_iter - 1][1] = (uint32_t)(ns - 1);
  ch[num_iter - 1][2] = start_hit; ch[num_iter - 1][3] = hit_num[ns - 1];
  *out = ch;
  *n_out = num_iter;
  return 0;
}

/* The chunk list of chunk_limits for tests: up to cap entries of
 * (start_seed, last_seed, start_hit, end_hit) into out[4 * cap]. */
int hzo_chunk_limits(const uint32_t *hit_num, uint64_t ns, uint32_t max_hits, uint32_t *out, uint32_t cap,
                     uint32_t *n_out) {
  if (ns == 0 || max_hits == 0) return HZO_E_INVALID;
  uint32_t(*ch)[4];
  uint32_t n;
  int rc = chunk_limits(hit_num, ns, max_hits, &ch, &n);
  if (rc) return rc;
  for (uint32_t i = 0; i < n && i < cap; i++)
    for (int k = 0; k < 4; k++) out[4 * i + k] = ch[i][k];
  *n_out = n;
  free(ch);
  return 0;
}

static int run_call(const hzo_target *t, const uint8_t *qry, uint32_t qlen, const uint64_t *seeds,
                    uint64_t ns, hsp_vec *out, hzo_stats *st) {
  const hzo_params *p = t->p;
  if (ns == 0) return 0;
  uint32_t *hit_num = malloc(ns * sizeof(uint32_t));
  if (!hit_num) return HZO_E_OOM;
  uint64_t acc = 0;
  for (uint64_t i = 0; i < ns; i++) {
    acc += hit_count(t, (uint32_t)(seeds[i] >> 32));
    if (acc > 0xFFFFFFFFull) { free(hit_num); return HZO_E_INVALID; } /* u32 num_hits */
    hit_num[i] = (uint32_t)acc;
  }
  uint32_t num_hits = (uint32_t)acc;
  st->seeds += ns;
  st->hits += num_hits;
  st->calls += 1;
  if (num_hits == 0) { free(hit_num); return 0; }

  /* chunk list: (start_seed, limit_pos, start_hit, end_hit) */
  uint32_t nchunks;
  uint32_t(*ch)[4];
  int crc = chunk_limits(hit_num, ns, p->max_hits, &ch, &nchunks);
  if (crc) { free(hit_num); return crc; }

  hsp_vec raw = {0};
  int rc = 0;
  for (uint32_t c = 0; c < nchunks && rc == 0; c++) {
    if (ch[c][3] - ch[c][2] == 0) continue;
    raw.n = 0;
    for (uint64_t s = ch[c][0]; s <= ch[c][1]; s++) {
      uint32_t k = (uint32_t)(seeds[s] >> 32);
      uint32_t cnt = hit_count(t, k);
      if (cnt == 0) continue;
      uint32_t b = k > 0 ? t->index_table[k - 1] : 0;
      uint32_t qloc = (uint32_t)(seeds[s] & 0xFFFFFFFFu) + t->sh->size;
      for (uint32_t j = 0; j < cnt; j++) {
        uint32_t rloc = t->pos_table[b + j] + t->sh->size;
        hzo_ext e = extend_hit(t->ref, t->rlen, qry, qlen, p, rloc, qloc);
        st->cells += e.cells;
        if (e.accepted && vec_push(&raw, e.hsp)) { rc = HZO_E_OOM; break; }
      }
      if (rc) break;
    }
    if (rc) break;
    st->raw_hsps += raw.n;
    uint64_t kept = hzo_dedup_and_order(raw.v, raw.n);
    for (uint64_t i = 0; i < kept; i++)
      if (vec_push(out, raw.v[i])) { rc = HZO_E_OOM; break; }
    st->hsps += kept;
  }
  free(raw.v);
  free(ch);
  free(hit_num);
  return rc;
}

/* One seed_and_filter call on the seeds chunk_seeds generates for [start,
 * end) of `qry` (fwd or rc codes).  *out is malloc'd. */
int hzo_seed_and_filter(const hzo_params *p, const hzo_shape *sh, const uint8_t *ref, uint64_t rlen,
                        const uint32_t *index_table, const uint32_t *pos_table, const uint8_t *qry,
                        uint64_t qlen, uint32_t start, uint32_t end, hzo_hsp **out, uint64_t *n_out,
                        hzo_stats *st) {
  *out = NULL;
  *n_out = 0;
  if (p->max_hits == 0 || rlen > 0xFFFFFFFFull || qlen > 0xFFFFFFFFull) return HZO_E_INVALID;
  if (end < start || (uint64_t)end + sh->size - 1 > qlen) return HZO_E_INVALID;
  hzo_target t = {p, sh, ref, (uint32_t)rlen, index_table, pos_table};
  uint64_t per = p->transitions ? 1 + sh->kmer_size : 1;
  uint64_t span = end - start;
  uint64_t *seeds = malloc((span * per + 1) * sizeof(uint64_t));
  if (!seeds) return HZO_E_OOM;
  uint64_t ns = gen_seeds(sh, p, qry, start, end, seeds);
  hsp_vec v = {0};
  int rc = run_call(&t, qry, (uint32_t)qlen, seeds, ns, &v, st);
  free(seeds);
  if (rc) { free(v.v); return rc; }
  *out = v.v;
  *n_out = v.n;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* The whole pass (run.rs:266-495): intervals x strands x WGA chunks.        */

/* intervals(): src/sequence.rs:322-334 (end inclusive). */
static uint64_t intervals_of(uint64_t block_len, uint32_t seed_size, uint32_t isz,
                             uint32_t (*out)[2]) {
  uint64_t n = 0;
  if (block_len <= seed_size) return 0;
  uint32_t end_pos = (uint32_t)(block_len - seed_size);
  uint64_t cur = 0;
  while (cur < end_pos) {
    uint64_t e = cur + isz < end_pos ? cur + isz : end_pos;
    if (out) { out[n][0] = (uint32_t)cur; out[n][1] = (uint32_t)e; }
    n++;
    cur += isz;
  }
  return n;
}

/* chunks(): src/seed.rs:488-496 ([i, min(i+wga, end+1)) while i < end). */
static uint64_t chunks_of(uint32_t start, uint32_t end, uint32_t wga, uint32_t (*out)[2]) {
  uint64_t n = 0;
  for (uint64_t i = start; i < end; i += wga) {
    uint64_t e = i + wga < (uint64_t)end + 1 ? i + wga : (uint64_t)end + 1;
    if (out) { out[n][0] = (uint32_t)i; out[n][1] = (uint32_t)e; }
    n++;
  }
  return n;
}

typedef struct {
  uint32_t interval, rev, start, end;
} hzo_batch;

/* batch list in run.rs order: per interval, plus chunks then minus chunks;
 * minus range = (qbl - end, qbl - start), qbl = block_len - seed_size. */
int64_t hzo_batches(uint64_t qlen, uint32_t seed_size, uint32_t interval, uint32_t wga,
                    uint32_t strand, hzo_batch *out) {
  uint64_t ni = intervals_of(qlen, seed_size, interval, NULL);
  uint32_t(*iv)[2] = malloc((ni ? ni : 1) * sizeof(*iv));
  if (!iv) return HZO_E_OOM;
  intervals_of(qlen, seed_size, interval, iv);
  uint32_t qbl = qlen > seed_size ? (uint32_t)(qlen - seed_size) : 0;
  int64_t n = 0;
  for (uint64_t i = 0; i < ni; i++) {
    for (int rev = 0; rev < 2; rev++) {
      if (!(strand & (1u << rev))) continue;
      uint32_t s = rev ? qbl - iv[i][1] : iv[i][0];
      uint32_t e = rev ? qbl - iv[i][0] : iv[i][1];
      uint64_t nc = chunks_of(s, e, wga, NULL);
      uint32_t(*cs)[2] = malloc((nc ? nc : 1) * sizeof(*cs));
      if (!cs) { free(iv); return HZO_E_OOM; }
      chunks_of(s, e, wga, cs);
      for (uint64_t c = 0; c < nc; c++) {
        if (out) {
          out[n].interval = (uint32_t)i; out[n].rev = (uint32_t)rev;
          out[n].start = cs[c][0]; out[n].end = cs[c][1];
        }
        n++;
      }
      free(cs);
    }
  }
  free(iv);
  return n;
}

typedef struct {
  uint32_t interval;
  uint32_t strand; /* 0 '+', 1 '-' */
  hzo_hsp h;
} hzo_out;

typedef struct {
  const hzo_target *t;
  const uint8_t *qf, *qr;
  uint32_t qlen;
  const hzo_batch *b;
  int64_t nb;
  hsp_vec *res;
  hzo_stats *st;
  int *rc;
  int64_t next;
  pthread_mutex_t mu;
} pass_ctx;

static void *pass_worker(void *arg) {
  pass_ctx *c = arg;
  const hzo_params *p = c->t->p;
  uint64_t per = p->transitions ? 1 + c->t->sh->kmer_size : 1;
  uint64_t *seeds = NULL;
  uint64_t seeds_cap = 0;
  for (;;) {
    pthread_mutex_lock(&c->mu);
    int64_t i = c->next++;
    pthread_mutex_unlock(&c->mu);
    if (i >= c->nb) break;
    const hzo_batch *b = &c->b[i];
    uint64_t need = (uint64_t)(b->end - b->start) * per + 1;
    if (need > seeds_cap) {
      free(seeds);
      seeds = malloc(need * sizeof(uint64_t));
      seeds_cap = seeds ? need : 0;
      if (!seeds) { c->rc[i] = HZO_E_OOM; continue; }
    }
    const uint8_t *q = b->rev ? c->qr : c->qf;
    uint64_t ns = gen_seeds(c->t->sh, p, q, b->start, b->end, seeds);
    c->rc[i] = run_call(c->t, q, c->qlen, seeds, ns, &c->res[i], &c->st[i]);
  }
  free(seeds);
  return NULL;
}

/* seed_and_filter_all over every batch of a query block, `threads` workers
 * over independent calls (each call is its own dedup scope set, so the
 * result does not depend on the thread count).  Output records are grouped
 * per interval: plus records then minus records, each in call order.
 * If max_batches > 0 only the first max_batches batches run (a bounded
 * sample for timing). */
int hzo_seed_and_filter_all(const hzo_params *p, const hzo_shape *sh, const uint8_t *ref,
                            uint64_t rlen, const uint32_t *index_table, const uint32_t *pos_table,
                            const uint8_t *qf, const uint8_t *qr, uint64_t qlen,
                            int64_t max_batches, hzo_out **out, uint64_t *n_out, hzo_stats *st) {
  *out = NULL;
  *n_out = 0;
  memset(st, 0, sizeof(*st));
  if (p->max_hits == 0 || rlen > 0xFFFFFFFFull || qlen > 0xFFFFFFFFull) return HZO_E_INVALID;
  int64_t nb = hzo_batches(qlen, sh->size, p->interval, p->wga_chunk, p->strand, NULL);
  if (nb < 0) return (int)nb;
  hzo_batch *b = malloc((nb ? nb : 1) * sizeof(hzo_batch));
  if (!b) return HZO_E_OOM;
  hzo_batches(qlen, sh->size, p->interval, p->wga_chunk, p->strand, b);
  if (max_batches > 0 && max_batches < nb) nb = max_batches;
  hzo_target t = {p, sh, ref, (uint32_t)rlen, index_table, pos_table};
  hsp_vec *res = calloc(nb ? nb : 1, sizeof(hsp_vec));
  hzo_stats *sts = calloc(nb ? nb : 1, sizeof(hzo_stats));
  int *rcs = calloc(nb ? nb : 1, sizeof(int));
  if (!res || !sts || !rcs) { free(b); free(res); free(sts); free(rcs); return HZO_E_OOM; }
  pass_ctx c;
  memset(&c, 0, sizeof(c));
  c.t = &t; c.qf = qf; c.qr = qr; c.qlen = (uint32_t)qlen; c.b = b; c.nb = nb;
  c.res = res; c.st = sts; c.rc = rcs; c.next = 0;
  pthread_mutex_init(&c.mu, NULL);
  uint32_t nt = p->threads ? p->threads : 1;
  if (nt > 256) nt = 256;
  pthread_t th[256];
  uint32_t started = 0;
  for (uint32_t i = 0; i + 1 < nt; i++)
    if (pthread_create(&th[started], NULL, pass_worker, &c) == 0) started++;
  pass_worker(&c);
  for (uint32_t i = 0; i < started; i++) pthread_join(th[i], NULL);
  pthread_mutex_destroy(&c.mu);

  int rc = 0;
  uint64_t total = 0;
  for (int64_t i = 0; i < nb; i++) {
    if (rcs[i] && !rc) rc = rcs[i];
    total += res[i].n;
    st->seeds += sts[i].seeds; st->hits += sts[i].hits; st->raw_hsps += sts[i].raw_hsps;
    st->hsps += sts[i].hsps; st->cells += sts[i].cells; st->calls += sts[i].calls;
  }
  hzo_out *o = NULL;
  if (rc == 0) {
    o = malloc((total ? total : 1) * sizeof(hzo_out));
    if (!o) rc = HZO_E_OOM;
  }
  if (rc == 0) {
    /* group per interval: plus batches first, then minus batches */
    uint64_t w = 0;
    int64_t i0 = 0;
    while (i0 < nb) {
      int64_t i1 = i0;
      while (i1 < nb && b[i1].interval == b[i0].interval) i1++;
      for (int pass = 0; pass < 2; pass++)
        for (int64_t i = i0; i < i1; i++) {
          if ((int)b[i].rev != pass) continue;
          for (uint64_t k = 0; k < res[i].n; k++) {
            o[w].interval = b[i].interval;
            o[w].strand = b[i].rev;
            o[w].h = res[i].v[k];
            w++;
          }
        }
      i0 = i1;
    }
    *out = o;
    *n_out = total;
  }
  for (int64_t i = 0; i < nb; i++) free(res[i].v);
  free(res); free(sts); free(rcs); free(b);
  return rc;
}

void hzo_free(void *ptr) { free(ptr); }
