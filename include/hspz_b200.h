/*
 * hspz_b200.h -- C ABI of the B200 seed-and-filter engine.
 *
 * Plain pointers and sizes only; every entry point returns 0 or a negative
 * HZ_E_* code and leaves a message in hz_last_error() (thread-local).  An
 * engine is single-threaded (like the reference's Engine, one per worker
 * thread) and owns all of its device memory.  There is no CPU fallback: on a
 * machine without a usable sm_100 device hz_engine_create fails with
 * HZ_E_CUDA.
 *
 * Each entry point names the reference interface it replaces (hspZ, Rust).
 */
#ifndef HSPZ_B200_H
#define HSPZ_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HZ_OK 0
#define HZ_E_STATE (-1)    /* call order violated (e.g. no query swapped in) */
#define HZ_E_CUDA (-5)     /* CUDA runtime error */
#define HZ_E_OOM (-12)     /* device or host allocation failed */
#define HZ_E_INVALID (-22) /* bad argument */
#define HZ_E_BUDGET (-28)  /* serving admission budget exceeded */
#define HZ_E_TIMEOUT (-110)

/* SegmentPair (src/hsp.rs:31-41): block-relative starts, extent, score. */
typedef struct hz_segment_pair {
  uint32_t ref_start;
  uint32_t query_start;
  uint32_t len;
  int32_t score;
} hz_segment_pair;

/* One record of a pass: LASTZ interval index, strand (0 '+', 1 '-'). */
typedef struct hz_pass_record {
  uint32_t interval;
  uint32_t strand;
  hz_segment_pair h;
} hz_pass_record;

/* EngineConfig (src/gpu/mod.rs:1005-1019) plus the run flags that
 * parameterise the path (src/cli.rs:41-183). */
typedef struct hz_config {
  int32_t sub_mat[64];   /* build_sub_mat (src/scoring.rs:41-120), device alphabet */
  char seed[64];         /* "12of19", "14of22" or a 1/0/T pattern (Shape::parse) */
  int32_t xdrop;         /* -x, 910 */
  int32_t hspthresh;     /* -H, 3000 */
  uint32_t noentropy;    /* -E */
  uint32_t transitions;  /* 1 unless --notransition */
  uint32_t step;         /* -e, seed-table step, 1 */
  uint32_t max_hits;     /* --max-hits; 0 derives 4194304 x device GiB (src/gpu/mod.rs:2422-2442) */
  uint32_t occ_cap;      /* per-seed occurrence cap, 0 = none (an extension of this build) */
  uint32_t wga_chunk;    /* -C, 250000 */
  uint32_t interval;     /* -I, 10000000 */
  uint32_t strand;       /* 1 plus, 2 minus, 3 both (-S) */
} hz_config;

/* Counters of one call or pass (FilterOutput, src/gpu/mod.rs:55-67). */
typedef struct hz_stats {
  uint64_t seeds;     /* seeds generated (valid windows x variants) */
  uint64_t hits;      /* seed hits expanded, after the occurrence cap */
  uint64_t raw_hsps;  /* HSPs above threshold before dedup */
  uint64_t hsps;      /* HSPs after dedup */
  uint64_t cells;     /* scalar X-drop cells scored, both directions */
  uint64_t calls;     /* seed_and_filter calls that had seeds */
} hz_stats;

typedef struct hz_engine hz_engine;

const char *hz_last_error(void);
void hz_free(void *p);

/* Shape::parse (src/seed.rs:49-79): width and care-position count. */
int hz_shape_info(const char *seed, uint32_t *size, uint32_t *kmer_size);

/* Engine::new minus the tables (src/gpu/mod.rs:1021-1128): binds `device`,
 * creates the engine's stream and loads the configuration. */
int hz_engine_create(const hz_config *cfg, int device, hz_engine **out);
void hz_engine_destroy(hz_engine *e);

/* Engine::new's tables as the reference builds them on the host
 * (EngineConfig.index_table / pos_table / ref_seq, src/gpu/mod.rs:1005-1011,
 * built by SeedTable::build_parallel src/seed.rs:207-363). ref_seq is in the
 * device alphabet. */
int hz_engine_load_tables(hz_engine *e, const uint32_t *index_table, uint64_t index_len,
                          const uint32_t *pos_table, uint64_t pos_len, const uint8_t *ref_seq,
                          uint64_t ref_len);

/* The same target built on the device from the ASCII reference block:
 * encode (src/sequence.rs:66-79) + SeedTable::build (src/seed.rs:135-180),
 * byte-identical tables, resident until the next load. */
int hz_engine_load_target(hz_engine *e, const uint8_t *ref_ascii, uint64_t len);

/* Copies the resident seed table back (tests / interop): index_len entries
 * of index_table and *pos_len of pos_table (pass NULL to query sizes). */
int hz_engine_read_tables(hz_engine *e, uint32_t *index_table, uint64_t *index_len, uint32_t *pos_table,
                          uint64_t *pos_len);

/* Engine::swap_query (src/gpu/mod.rs:1142-1148): both strands already in
 * the device alphabet. */
int hz_swap_query(hz_engine *e, const uint8_t *query, const uint8_t *query_rc, uint64_t len);

/* swap_query from the ASCII query block: the forward and reverse-complement
 * encodings are made on the device (src/sequence.rs:66-86, 212-230). */
int hz_swap_query_ascii(hz_engine *e, const uint8_t *query_ascii, uint64_t len);

/* Engine::upload_seeds (src/gpu/mod.rs:1246): seeds kmer << 32 | position. */
int hz_upload_seeds(hz_engine *e, uint32_t slot, const uint64_t *seeds, uint64_t n);

/* Engine::generate_seeds (src/gpu/mod.rs:1312-1463): the seeds of query
 * positions [start, end) of one strand, made and looked up on the device;
 * *n_seeds as chunk_seeds would return. */
int hz_generate_seeds(hz_engine *e, uint32_t slot, int rev, uint32_t start, uint32_t end, int transitions,
                      uint64_t *n_seeds);

/* Engine::seed_and_filter (src/gpu/mod.rs:1499-2178): lookup, MAX_HITS
 * chunking, expansion, X-drop extension, entropy, and per-chunk
 * dedup_and_order; *out (hz_free) is deduped per chunk, LASTZ order,
 * concatenated.  HZ_E_STATE without a swapped-in query. */
int hz_seed_and_filter(hz_engine *e, uint32_t slot, int rev, hz_segment_pair **out, uint64_t *n,
                       hz_stats *stats);

/* seed_and_filter_all (src/run.rs:266-495), plain per-chunk form: every
 * interval x strand x WGA chunk of the swapped-in query, one launch chain per
 * call.  Records are grouped per interval, plus before minus, in call order.
 * By default the calls run on four workspaces at once (tuning knob
 * "plain_streams"); the records do not depend on it. */
int hz_run_pass(hz_engine *e, hz_pass_record **out, uint64_t *n, hz_stats *stats);

/* One query block for the batched form (ASCII, records joined by '&'). */
typedef struct hz_query {
  const uint8_t *ascii;
  uint64_t len;
} hz_query;

/* One record of a batched run: query index, interval, strand, HSP. */
typedef struct hz_batch_record {
  uint32_t query;
  uint32_t interval;
  uint32_t strand;
  hz_segment_pair h;
} hz_batch_record;

/* Replaces the resident query store with `nq` query blocks (the reference
 * swaps one query bin at a time, src/gpu/mod.rs:1142-1148; this keeps many
 * resident).  Both strands are encoded on the device. */
int hz_stage_queries(hz_engine *e, const hz_query *queries, uint32_t nq);

/* Makes staged query `index` the one that swap_query would have put in place
 * (the target of hz_generate_seeds / hz_upload_seeds / hz_seed_and_filter /
 * hz_run_pass), without another upload. */
int hz_select_query(hz_engine *e, uint32_t index);

/* Batched form of seed_and_filter_all (src/run.rs:266-495) over every staged
 * query: all calls of many queries go through shared waves (one lookup, one
 * persistent gate launch over a device work queue, one read-back per wave)
 * instead of one launch chain per call.  Records are grouped by query, then
 * exactly as hz_run_pass orders them; each query's records equal what
 * hz_run_pass returns for that query alone.  The engine keeps the host
 * buffer it assembles the records in (20 bytes per record) until it is
 * destroyed, so a repeated pass does not allocate it again. */
int hz_run_batched(hz_engine *e, hz_batch_record **out, uint64_t *n, hz_stats *stats);

/* One line of a .segments file (hsp::Record, src/hsp.rs:179-187): the
 * chromosome indices into the reference and query tables and the 1-based,
 * chromosome-relative coordinates (end = start + length). */
typedef struct hz_segment_record {
  uint32_t r_chr;
  uint32_t q_chr;
  uint64_t r_start;
  uint64_t r_end;
  uint64_t q_start;
  uint64_t q_end;
  int32_t score;
  uint32_t pad;
} hz_segment_record;

/* render_records (src/hsp.rs:234-252): the text of a .segments file, one
 * tab-separated line per record -- reference name, start, end, query name,
 * start, end, strand ('+' or '-'), score.  Names are NUL-terminated; *out is
 * NUL-terminated, *out_len excludes the NUL, freed with hz_free.  A host-only
 * entry point (no device needed). */
int hz_render_records(const hz_segment_record *recs, uint64_t n, const char *const *r_names, uint32_t nr,
                      const char *const *q_names, uint32_t nq, char strand, char **out, uint64_t *out_len);

/* dedup_and_order (src/hsp.rs:94-126) on host records, in place; returns
 * the kept count in *n_out. */
int hz_dedup_and_order(hz_segment_pair *h, uint64_t n, uint64_t *n_out);

/* No counterpart in the reference.  dedup_and_order of one set of HSPs that
 * already sits in device memory, for callers that cannot allocate device
 * memory themselves or let a library do it -- e.g. a host whose own
 * allocator owns the whole device, or a serving loop that admits work
 * against a fixed memory budget.  It allocates nothing: its working memory is
 * a fixed array of about 6 MB compiled into this library, which every GPU
 * that loads the library holds until the process exits.
 *   d_in:    n records on the current device (4-byte aligned), read only;
 *            n <= HZ_NOALLOC_MAX_HSPS, larger n is refused with HZ_E_INVALID.
 *   d_out:   room for n records; receives the kept records in LASTZ order.
 *   d_n_out: one device uint32, receives the kept count.
 *   stream:  a cudaStream_t (NULL for the default stream).
 * d_in, d_out and d_n_out must not overlap (no in-place dedup); overlapping
 * buffers are refused with HZ_E_INVALID.
 * The work is queued on `stream` and the call returns at once; results are
 * valid once the stream reaches that point.  The first call in a device's
 * context looks up the scratch array's device address, so make it before
 * any stream capture; a process that resets the device (cudaDeviceReset)
 * gets a new context, and its next call looks the address up again, so that
 * call too belongs outside a capture.  All calls share the one scratch
 * array: calls whose work overlaps on the GPU (other streams, other host
 * threads) race and corrupt each other's results, so keep them ordered on
 * one stream. */
#define HZ_NOALLOC_MAX_HSPS (1u << 18)
int hz_dedup_and_order_device_noalloc(const hz_segment_pair *d_in, uint32_t n, hz_segment_pair *d_out,
                                      uint32_t *d_n_out, void *stream);

/* Per-kernel device time (CUDA events on the engine's stream) since the last
 * reset; enable with hz_engine_set_profiling.  Entry i: name, total ms,
 * launches.  Returns HZ_E_INVALID past the last entry. */
int hz_engine_set_profiling(hz_engine *e, int on);
int hz_engine_profile_entry(hz_engine *e, uint32_t i, char *name, uint32_t name_cap, double *ms,
                            uint64_t *launches);
int hz_engine_profile_reset(hz_engine *e);

/* Launch-shape knobs (no reference counterpart; results never depend on
 * them): "gate_version" (2, the default: the lockstep gate over 2-bit packed
 * sequences, used whenever every ACGT score fits a signed byte; 1: the
 * lane-refill gate over 8-bit codes, which also serves wider scores),
 * "gate_sparse" (the lockstep gate's tile setup: -1, the default, chosen
 * from the target's average bucket; 0 a lane per (position, seed) pair;
 * 1 a lane per position, for targets whose tiles span many positions),
 * "gate_tile" (hits per gate warp tile: 64, 128, 256),
 * "gate_cap" (cells per direction before a hit leaves the gate as a long
 * candidate -- for the lane-per-candidate long kernel after the lockstep
 * gate, for the warp kernel after the lane-refill gate -- multiple of 8,
 * 8..65528), "gate_blocks_per_sm" (0 = occupancy maximum),
 * "wave_positions" (seed positions per batched wave), "wave_hits_cap" (a
 * batched wave of several calls holding more seed hits than this, default
 * 2^33, is run again as smaller waves, which bounds the hit-dependent wave
 * buffers on repeat-dense input), "device_dedup" (1: the
 * batched form dedups on the device, and so does a plain-form call holding at
 * least "device_dedup_min" raw HSPs (default 65536); 0: every dedup on the
 * host, as the reference does),
 * "graph" (1: the batched form captures each wave's kernel chain as a CUDA
 * graph and replays it, updating the instantiated graph in place),
 * "plain_streams" (1..4, default 4: hz_run_pass runs its calls on this
 * engine and plain_streams - 1 more workspaces over the same target, each
 * with its own host thread and stream, so one call's read-back and host dedup
 * overlap other calls' kernels; 1: one call at a time on this engine; an
 * engine given a caller's stream by hz_engine_set_stream runs every call on
 * that stream.  Each extra workspace is made on first use and holds its own
 * grow-only wave buffers -- about as much device memory as the largest call
 * it has run needs, i.e. up to plain_streams times one engine's wave memory
 * in all -- until the engine is destroyed or plain_streams is lowered, which
 * frees the workspaces beyond the new count.  A workspace that runs out of
 * device memory hands its call to this engine and is freed; the pass goes on),
 * "tile_cap" / "cand_cap" / "raw_cap" (starting capacities of the gate's
 * tile table, the candidate list and the raw-HSP list; a wave that needs more
 * grows them and runs again; the extra workspaces start from at least this
 * engine's capacities). */
int hz_engine_set_tuning(hz_engine *e, const char *key, int64_t value);

/* Autotuner (no reference counterpart).  Times the batched form on a
 * sample of the staged work -- every k-th call, up to sample_positions seed
 * positions (0 = 2^24) -- under each candidate launch shape and keeps the
 * fastest: gate_tile (hits a gate warp stages per tile: 64, 128, 256, i.e.
 * 2..8 per lane), gate_cap (cells a lane scores before a hit moves to the warp
 * kernel: 64..1024) and graph (the wave chain replayed as a CUDA graph or
 * launched kernel by kernel).  Results never depend on the choice. */
typedef struct hz_tuning {
  int32_t gate_tile;
  int32_t gate_cap;
  int32_t gate_blocks_per_sm;
  int32_t graph;
  double best_ms;           /* sample time with the chosen shape */
  double start_ms;          /* sample time with the shape in place before */
  uint32_t candidates;
  uint32_t sample_calls;
  uint64_t sample_positions;
} hz_tuning;
int hz_engine_autotune(hz_engine *e, uint64_t sample_positions, hz_tuning *out);

/* Kernel launches issued by this engine since creation, its serving
 * workers' included. */
uint64_t hz_engine_launches(hz_engine *e);

/* Runs the engine's work on a caller-owned cudaStream_t (NULL restores the
 * engine's own stream), so callers can order and time it with their events. */
int hz_engine_set_stream(hz_engine *e, void *stream);

/* ---- serving loop ------------------------------------------------------
 * The reference runs one bin of queries at a time (run_bins,
 * src/run.rs:816-887) and has no request queue; these entry points keep a
 * target resident and take query blocks as they arrive.  hz_serve_start
 * starts `workers` host threads, each with its own query store, wave buffers
 * and stream over the engine's target tables.  A free worker takes the queued
 * requests in arrival order (at most `max_batch_queries` of them, 0 = 64) and
 * runs them as one batched pass, so requests that arrive while others run
 * join the next batch.  A request's records equal what hz_run_pass returns
 * for that query block alone.
 * Admission by memory: every worker holds device memory -- its grow-only
 * query store, wave and dedup buffers -- and counts against `budget_bytes`
 * with what it measurably holds while idle, or, while it runs a batch, the
 * larger of that and the batch's estimate (hz_serve_estimate per request).
 * A batch is formed only while the sum over all workers stays within the
 * budget.  A worker whose buffers outgrow the budget after a batch frees
 * them; idle workers free theirs when a queued request could not fit
 * otherwise.  The estimates grow with the hits per position, candidates and
 * raw HSPs per hit the loop has seen, so a request accepted by
 * hz_serve_submit may later estimate above the whole budget; it then runs
 * alone once no other worker holds memory.
 * Failures: if a batch fails, each of its requests runs again alone, so only
 * a request that fails by itself reports an error. */
typedef struct hz_serve_config {
  uint64_t budget_bytes;       /* device working memory for requests in flight */
  uint32_t workers;            /* 1..8 */
  uint32_t max_batch_queries;  /* 0 = 64 */
} hz_serve_config;

typedef struct hz_serve_times {
  double queued_ms;        /* submit -> taken by a worker */
  double service_ms;       /* taken -> its batch finished */
  double total_ms;         /* submit -> finished */
  uint32_t batch_queries;  /* queries in the batch it ran in */
  uint32_t worker;         /* index of the worker that ran it */
} hz_serve_times;

/* HZ_E_STATE if a loop already runs or no target is loaded.  While the loop
 * runs, the engine's own entry points that touch the target are refused. */
int hz_serve_start(hz_engine *e, const hz_serve_config *cfg);
/* Copies the query block; HZ_E_BUDGET if its estimated working memory alone
 * exceeds the budget (it could never be admitted). */
int hz_serve_submit(hz_engine *e, const uint8_t *ascii, uint64_t len, uint64_t *ticket);
/* Waits up to timeout_ms (< 0: without limit) for the ticket.  HZ_E_TIMEOUT
 * if it has not finished (the ticket stays valid); otherwise the ticket is
 * consumed and either *out holds its records (hz_pass_record, freed with
 * hz_free) or the call returns the request's own error (HZ_E_STATE for a
 * cancelled one).  HZ_E_INVALID for an unknown or consumed ticket. */
int hz_serve_poll(hz_engine *e, uint64_t ticket, int timeout_ms, hz_pass_record **out, uint64_t *n,
                  hz_serve_times *times);
/* The device working memory the loop currently expects a request of `len`
 * bases to need (the figure admission and hz_serve_submit use). */
int hz_serve_estimate(hz_engine *e, uint64_t len, uint64_t *bytes);
/* Totals (seeds, hits, cells, HSPs, calls) over every batch finished since
 * hz_serve_start, and the requests still queued or running. */
int hz_serve_stats(hz_engine *e, hz_stats *stats, uint64_t *queued, uint64_t *running);
/* Cancels a request that no worker has taken yet (HZ_E_STATE otherwise). */
int hz_serve_cancel(hz_engine *e, uint64_t ticket);
/* Finishes every queued request, joins the workers and frees their memory.
 * Tickets not polled before the stop are dropped.  No other serving entry
 * point may run on the engine while it stops. */
int hz_serve_stop(hz_engine *e);

#ifdef __cplusplus
}
#endif
#endif
