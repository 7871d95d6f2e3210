/*
 * sumcheck_b200.h -- C ABI of the B200 SumCheck prover (libsumcheck_b200.so).
 *
 * Plain C: pointers, sizes and status codes; no CUDA, torch or C++ types. Every call
 * returns SC_OK (0) or an SC_ERR_* code; sc_last_error() gives the message of the
 * calling thread's last failure. Device work runs on the stream given to sc_ctx_create.
 *
 * The reference (snarang181/sumcheck-triton) exposes this path two ways, and nothing
 * here is a binding of its code: its Python API `zkduel.sumcheck(eval_tables, q,
 * expression, challenges, num_rounds, bit_width, backend)` (src/zkduel/api.py:26-64)
 * and its CUDA executable's round loop (cuda/src/field_sumcheck.cu:1012-1088, CLI
 * :1091-1176). Each entry point below names the reference interface it replaces.
 *
 * Data formats
 *   field element  L little-endian u32 limbs, L in {1, 2, 4, 8}; "Montgomery" means the
 *                  limbs of x * 2^(32 L) mod p, always fully reduced (< p).
 *   tables         limb-planar device memory: table k, limb l is the u32 plane
 *                  tables[(k * L + l) * 2^n + i], i < 2^n. Device pointer, 16-byte aligned.
 *   expression     sum of terms coeff * prod(tables): term i has term_lens[i] factors
 *                  flat[term_offsets[i] ...], each a table index < num_vars.
 */
#ifndef SUMCHECK_B200_H
#define SUMCHECK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SC_OK 0
#define SC_ERR_INVALID 1        /* bad argument (sizes, alignment, NULL, ranges)        */
#define SC_ERR_UNSAFE_MODULUS 2 /* modulus outside the Montgomery product's exactness   */
#define SC_ERR_CUDA 3           /* a CUDA runtime call failed                            */
#define SC_ERR_UNSUPPORTED 4    /* outside the compiled limits (degree, tables, terms)  */
#define SC_ERR_DEVICE 5         /* the device reported an error status (see sc_prove_resume) */
#define SC_ERR_NOMEM 6          /* device or host allocation failed                     */
#define SC_ERR_TIMEOUT 7        /* a bounded wait ran out (sc_server_wait / _drain)     */
#define SC_ERR_PENDING 8        /* the request has not completed yet                    */
#define SC_SUSPENDED 9          /* the request was suspended; its transcript is readable */

#define SC_CHALLENGE_SHA3 0     /* r_j = SHA3 transcript rule (field_sumcheck.cu:857-907) */
#define SC_CHALLENGE_FIXED 1    /* r_j = 1 (field_sumcheck.cu:1058)                       */
#define SC_CHALLENGE_EXPLICIT 2 /* r_j given by the caller (api.py:26-35 `challenges`)    */

#define SC_TABLE_UNIFORM 0      /* uniform in [0, p): counter-based SplitMix64 + rejection */
#define SC_TABLE_BERNOULLI 1    /* 0/1 selectors                                           */
#define SC_TABLE_ARITH 2        /* SC_TABLE_ARITH + v: the reference's fill of table v     */
                                /* (seed + 7919 (v+1) + 104729 (off+1)) mod p,             */
                                /* field_sumcheck.cu:123-128, :593-611                     */

#define SC_MAX_LIMBS 8
#define SC_MAX_DEGREE 7         /* 8 interpolation points, field_sumcheck.cu:29 */
#define SC_MAX_VARS 32
#define SC_MAX_TERMS 32
#define SC_MAX_FACTORS 128      /* total factors over all terms */
#define SC_MAX_ROUNDS 40

typedef struct sc_ctx sc_ctx;
typedef struct sc_field sc_field;
typedef struct sc_expr sc_expr;

/* Library version (major * 10000 + minor * 100 + patch). */
int sc_version(void);

/* Message of the calling thread's last failed call ("" if none). */
const char* sc_last_error(void);

/* A prover context on `device`, issuing all work on `stream` (a cudaStream_t; NULL for
 * the legacy default stream). Owns the scratch buffers (fold ping-pong, block partials,
 * proof state), grown on demand. One context per host thread.
 * Replaces: the CUDA executable's per-run setup (field_sumcheck.cu:1178-1225). */
int sc_ctx_create(int device, void* stream, sc_ctx** out);
int sc_ctx_destroy(sc_ctx* ctx);
/* Waits for all work of the context's stream. */
int sc_ctx_synchronize(sc_ctx* ctx);
/* Per-launch device timing of the round kernels (CUDA events on the context's stream),
 * off by default. sc_ctx_launch_times sets *count to the number of recorded launch
 * durations (ms, issue order, for launches completed by the last synchronising call) and
 * moves the first min(count, capacity) of them into out_ms (NULL: only counts). The reference's equivalent is its
 * --timing-mode round-sum / --timer events (field_sumcheck.cu:1032-1080, :1237-1246). */
int sc_ctx_set_timing(sc_ctx* ctx, int enable);
int sc_ctx_launch_times(sc_ctx* ctx, float* out_ms, int capacity, int* count);

/* A field of modulus p (L limbs) with nprime = -p^-1 mod 2^32. Rejects, with
 * SC_ERR_UNSAFE_MODULUS, the moduli the reference's guard rejects: even or < 3, wrong
 * nprime, or outside (2p-1) + (p-1)(2^32-1) < 2^(32(L+1)).
 * Replaces: zkduel.fields.FieldSpec / check_montgomery_modulus (src/zkduel/fields.py:190-255)
 * and the executable's FIELDS table (field_sumcheck.cu:39-121). */
int sc_field_init(int limbs, const uint32_t* modulus, uint32_t nprime, sc_field** out);
int sc_field_destroy(sc_field* field);

/* A constraint expression. coeffs[i] is term i's integer coefficient; if coeff_limbs is
 * not NULL it overrides coeffs with non-negative 8-limb values (num_terms x 8 u32), for
 * coefficients beyond int64 (the caller reduces them mod p).
 * Replaces: encode_expression_with_coeffs (src/zkduel/_expr.py:87-110) and the
 * executable's per-workload templates (field_sumcheck.cu:389-590). */
int sc_expr_compile(int num_vars, int num_terms, const int64_t* coeffs,
                    const uint32_t* coeff_limbs, const int32_t* term_lens,
                    const int32_t* term_offsets, const int32_t* flat, sc_expr** out);
int sc_expr_destroy(sc_expr* expr);
int sc_expr_degree(const sc_expr* expr);
int sc_expr_num_vars(const sc_expr* expr);

/* Fills num_tables tables of 2^num_rounds entries (Montgomery, limb-planar) at tables_dev.
 * kinds[k] is SC_TABLE_UNIFORM, SC_TABLE_BERNOULLI or SC_TABLE_ARITH + v.
 * Replaces: fill_tables_kernel (field_sumcheck.cu:593-611) and the Triton _make_tables
 * (benchmarks/field_sweep/triton_sweep.py:425-452). Asynchronous. */
int sc_tables_generate(sc_ctx* ctx, const sc_field* field, int num_tables, int num_rounds,
                       const int32_t* kinds, uint64_t seed, uint32_t* tables_dev);

/* In-place conversion of num_tables x L planes of `entries` values between canonical
 * form (< p) and Montgomery form. Asynchronous.
 * Replaces: the Triton backend's host Montgomery encode/decode
 * (src/zkduel/triton_backend/u256_sumcheck.py:99-109). */
int sc_tables_to_mont(sc_ctx* ctx, const sc_field* field, uint32_t* tables_dev,
                      uint64_t entries, int num_tables);
int sc_tables_from_mont(sc_ctx* ctx, const sc_field* field, uint32_t* tables_dev,
                        uint64_t entries, int num_tables);

/* Element-wise field arithmetic on device arrays of count elements (element-major, L words
 * each, values < p): op 0 = Montgomery product a b R^-1, 1 = a + b, 2 = a - b (mod p).
 * Exposes the prover's own device arithmetic for checking against big integers.
 * Replaces: the Triton backend's elementwise uint256 kernels
 * (src/zkduel/triton_backend/uint256.py:1149-1313). Asynchronous. */
int sc_field_apply(sc_ctx* ctx, const sc_field* field, int op, const uint32_t* a_dev,
                   const uint32_t* b_dev, uint32_t* out_dev, uint64_t count);

/* Measures the device's 32-bit integer multiply-add rate (IMAD/s) with a probe kernel of
 * independent mad.lo / mad.hi chains (the instruction pair of the Montgomery product);
 * the denominator of the integer-pipe roofline. Synchronous, about a millisecond.
 * No counterpart in the reference (it reports no roofline). */
int sc_calibrate_imad(sc_ctx* ctx, double* out_imad_per_s);

/* One SumCheck proof over num_rounds variables: num_rounds launches, no host round trip,
 * then one copy of the results to the host (the call returns when they are there).
 *   tables_dev           num_vars tables of 2^num_rounds entries, Montgomery, limb-planar;
 *                        read only.
 *   challenge_mode       SC_CHALLENGE_*; explicit_challenges (host, num_rounds x L,
 *                        Montgomery) is read only in SC_CHALLENGE_EXPLICIT mode.
 * Outputs (host, Montgomery limbs; any may be NULL):
 *   out_round_polys      num_rounds x (degree + 1) x L: g_j(0..degree)
 *   out_challenges       num_rounds x L: r_j (r_{n-1} is the final-point challenge)
 *   out_finals           (1 + num_vars) x L: g_{n-1}(r_{n-1}), then f_k(r_0..r_{n-1})
 *   out_claim0           L: g_0(0) + g_0(1), the sum over the hypercube
 *   out_checksum         sum over rounds and points of sum_i (i + 1) limb_i
 * Replaces: zkduel.sumcheck (src/zkduel/api.py:26-64) and run_once
 * (field_sumcheck.cu:1012-1088). */
int sc_prove(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int num_rounds,
             const uint32_t* tables_dev, int challenge_mode, const uint32_t* explicit_challenges,
             uint32_t* out_round_polys, uint32_t* out_challenges, uint32_t* out_finals,
             uint32_t* out_claim0, uint64_t* out_checksum);

/* How sc_prove runs this proof: *out_launches kernel launches (the per-launch timings of
 * sc_ctx_launch_times come in this number per proof). Rounds before *out_tail_round take a
 * launch each; from it on (when < num_rounds), the rounds are small enough for one block,
 * and one launch proves them all, round after round inside that block. No counterpart in
 * the reference (its executable launches per round and per point). */
int sc_prove_launches(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int num_rounds,
                      int* out_launches, int* out_tail_round);

/* sc_prove without any allocation, for callers that cannot call cudaMalloc (code inside
 * another framework's memory pool or under a fixed device-memory budget, plug-ins that may
 * not grow the process's footprint after start-up). No counterpart in the reference.
 * Same arguments and outputs as sc_prove (outputs are written straight into the caller's
 * host arrays). Its scratch is one 32 MiB array in device memory that every GPU loading
 * the library holds until exit; proofs needing more (about K L 2^n 3 bytes of fold
 * buffers plus under 1 MiB) fail with SC_ERR_UNSUPPORTED before anything runs. The first
 * call on a device looks up that array's device address: make it before any stream
 * capture, and do not reset the device's primary context (cudaDeviceReset) after it.
 * Synchronous: returns once the results are in the caller's arrays. Calls share the
 * array: calls that overlap on one GPU race, so issue them on one stream or one after
 * another. */
int sc_prove_noalloc(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int num_rounds,
                     const uint32_t* tables_dev, int challenge_mode,
                     const uint32_t* explicit_challenges, uint32_t* out_round_polys,
                     uint32_t* out_challenges, uint32_t* out_finals, uint32_t* out_claim0,
                     uint64_t* out_checksum);

/* ---------------------------------------------------------------- batched proving
 *
 * A batch holds `count` independent proofs over one field: proof i proves expression
 * exprs[i] over num_rounds[i] variables on the device tables tables_dev[i] (layout as for
 * sc_prove; read only; they must stay allocated while the batch exists). Round t of every
 * proof runs in one persistent launch ("tick") whose blocks pull (proof, tile) items from a
 * device work queue; the whole batch is one CUDA graph, replayed by every sc_batch_run.
 * Challenges: SC_CHALLENGE_SHA3 or SC_CHALLENGE_FIXED. threads (32..256, multiple of 32)
 * and pairs_per_thread (1..64) set the tile (threads x pairs_per_thread pairs per item);
 * 0 picks the defaults (256, 2). Results are bit-identical to sc_prove of each proof alone.
 * No counterpart in the reference, which proves one proof at a time
 * (cuda/src/field_sumcheck.cu:1012-1088; src/zkduel/api.py:26-64). */
typedef struct sc_batch sc_batch;
int sc_batch_create(sc_ctx* ctx, const sc_field* field, int count, const sc_expr* const* exprs,
                    const int32_t* num_rounds, const uint32_t* const* tables_dev,
                    int challenge_mode, int threads, int pairs_per_thread, sc_batch** out);
/* The same with tiles chosen per degree class and per proof (what the autotuner drives):
 * class_threads[3] = threads per block of the degree classes <= 2, <= 4, <= 7 (0: default);
 * proof_pairs_per_thread[count] = each proof's tile, threads x pairs_per_thread pairs per
 * work item (0: 2). Either array may be NULL (all defaults). No counterpart in the reference,
 * as sc_batch_create. */
int sc_batch_create_tiled(sc_ctx* ctx, const sc_field* field, int count, const sc_expr* const* exprs,
                          const int32_t* num_rounds, const uint32_t* const* tables_dev,
                          int challenge_mode, const int32_t* class_threads,
                          const int32_t* proof_pairs_per_thread, sc_batch** out);
/* Enqueues one run after the work queued on the context's stream (the context's stream
 * then waits for it). Asynchronous. */
int sc_batch_run(sc_batch* batch);
/* sc_batch_run in two halves, so that batches sharing a context overlap on the device:
 * sc_batch_launch enqueues the run after the work queued on the context's stream and returns;
 * sc_batch_join makes the context's stream wait for that run. Launch every batch, then join
 * every batch. */
int sc_batch_launch(sc_batch* batch);
int sc_batch_join(sc_batch* batch);
/* Waits for the last run; its results are then readable with sc_batch_result. */
int sc_batch_wait(sc_batch* batch);
/* Outputs of proof `index` of the last run, laid out as sc_prove's. */
int sc_batch_result(sc_batch* batch, int index, uint32_t* out_round_polys,
                    uint32_t* out_challenges, uint32_t* out_finals, uint32_t* out_claim0,
                    uint64_t* out_checksum);
/* Outputs of every proof of the last run in one call: proof 0's arrays, then proof 1's, and
 * so on, each laid out as sc_prove's (out_round_polys holds sum_p n_p (d_p + 1) L words,
 * out_challenges sum_p n_p L, out_finals sum_p (1 + K_p) L, out_claim0 count x L,
 * out_checksums count). Any may be NULL. */
int sc_batch_results(sc_batch* batch, uint32_t* out_round_polys, uint32_t* out_challenges,
                     uint32_t* out_finals, uint32_t* out_claim0, uint64_t* out_checksums);
/* A batch splits its proofs by degree class (degree <= 2, <= 4, <= 7); each class runs
 * its own sequence of ticks on its own stream. sc_batch_classes gives each class's degree
 * bound and tick count; sc_batch_class_proofs the indices of its proofs. */
int sc_batch_classes(sc_batch* batch, int32_t* out_degree_class, int32_t* out_ticks, int capacity,
                     int* count);
int sc_batch_class_proofs(sc_batch* batch, int cls, int32_t* out_indices, int capacity, int* count);
/* Start and end of every tick of the last run, in ms from the run's start (CUDA events
 * recorded inside the graph around each launch), class after class in sc_batch_classes
 * order, available after sc_batch_wait. Classes overlap in time; a kernel's duration is
 * end - start. Only the first `capacity` are copied; *count is the number of ticks. */
int sc_batch_tick_times(sc_batch* batch, float* out_start_ms, float* out_end_ms, int capacity,
                        int* count);
int sc_batch_destroy(sc_batch* batch);

/* ---- One proof split across ranks ----------------------------------------------------
 * Replaces: nothing; the reference proves on one device (cuda/src/field_sumcheck.cu:1012-1088).
 *
 * With world = 2^w ranks, rank r holds entries [r C, (r + 1) C), C = 2^(num_rounds - w), of
 * every table (limb-planar, C entries per plane). Protocol, identical on every rank:
 *   for j in 0 .. sc_split_local_rounds() - 1:
 *     sc_split_round(j, share)            this rank's share of g_j(0..d): (d + 1) L words
 *     all-gather the shares (rank order)  (the caller's collective, e.g. NCCL)
 *     sc_split_commit(j, shares)          sum, checksum, SHA3 challenge, claim (on the device)
 *   sc_split_last_entries(entries)        this rank's chunk folded to one entry per table (K L)
 *   all-gather the entries (rank order)
 *   sc_split_finish(all_entries)          the last w rounds on the W-entry tables
 *   sc_split_result(...)                  as sc_prove's outputs; the same on every rank and
 *                                         bit-identical to sc_prove on the whole tables.
 * With world = 1 the protocol is a whole proof (sc_split_finish(NULL)). */
typedef struct sc_split sc_split;
int sc_split_create(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int num_rounds, int world,
                    int rank, const uint32_t* local_tables_dev, int challenge_mode, sc_split** out);
int sc_split_local_rounds(const sc_split* split);
int sc_split_round(sc_split* split, int round, uint32_t* out_share);
int sc_split_commit(sc_split* split, int round, const uint32_t* shares);
int sc_split_last_entries(sc_split* split, uint32_t* out_entries);
int sc_split_finish(sc_split* split, const uint32_t* all_entries);
int sc_split_result(sc_split* split, uint32_t* out_round_polys, uint32_t* out_challenges,
                    uint32_t* out_finals, uint32_t* out_claim0, uint64_t* out_checksum);
int sc_split_destroy(sc_split* split);

/* ---- Transcripts: suspending and resuming a proof ----------------------------------
 * No counterpart in the reference: its proofs run start to finish inside one call.
 *
 * A transcript is a proof stopped at a round boundary: a flat array of u32 words that a
 * caller may store anywhere (file, database, another process) and later continue from the
 * same tables, on any context or server of the same field, with results bit-identical to
 * the uninterrupted proof. Layout (little-endian words):
 *   0  magic 0x31524353 ("SCR1")     1  header words (16)    2  limbs L
 *   3  num_rounds n                  4  num_vars K            5  degree d
 *   6  challenge mode                7  rounds done j (0..n)
 *   8  expression digest (u64)      10  field digest (u64)   12  tables tag (u64)
 *  14  state words S                15  0
 *  16  state: [0] 0, [1] device status, [2..3] checksum so far (u64), then
 *      g_0..g_{n-1}   n x 8 x L     (slot t of round i: g_i(t); rounds < j filled)
 *      r_0..r_{n-1}   n x L
 *      finals         (1 + K) x L   (when j = n)
 *      claim0         L
 *      claim          L             (g_{j-1}(r_{j-1}), the claim round j meets)
 * S = 4 + L (9 n + K + 3); sc_transcript_words() = 16 + S.
 * The digests bind a transcript to its field and expression; the tables tag is the
 * caller's name for the tables (sc_tables_tag for seeded ones; any value otherwise) and
 * is carried, not checked, by sc_prove_resume. Resuming folds the tables up to round j
 * with the recorded challenges (about one pass over them), then proves on. */
int sc_transcript_words(const sc_field* field, const sc_expr* expr, int num_rounds, uint64_t* out_words);
/* A transcript with no rounds done (the caller's `words`-word array). */
int sc_transcript_init(const sc_field* field, const sc_expr* expr, int num_rounds, int challenge_mode,
                       uint64_t tables_tag, uint32_t* transcript, uint64_t words);
/* Header of a transcript (checked for consistency); any output may be NULL. Host only. */
int sc_transcript_info(const uint32_t* transcript, uint64_t words, int* out_num_rounds,
                       int* out_rounds_done, int* out_challenge_mode, uint64_t* out_tables_tag);
/* Outputs of a complete transcript, laid out as sc_prove's; SC_ERR_PENDING before that. */
int sc_transcript_result(const sc_field* field, const sc_expr* expr, const uint32_t* transcript,
                         uint64_t words, uint32_t* out_round_polys, uint32_t* out_challenges,
                         uint32_t* out_finals, uint32_t* out_claim0, uint64_t* out_checksum);
/* The tag of tables generated by sc_tables_generate(num_tables, table_kinds, seed): what
 * the server records in its requests' transcripts and checks on resume. Host only. */
int sc_tables_tag(int num_tables, const int32_t* table_kinds, uint64_t seed, uint64_t* out_tag);
/* Proves rounds [rounds done, stop_round) of the transcript's proof on tables_dev (T_0,
 * as for sc_prove) and updates the transcript in place; stop_round = num_rounds completes
 * it. Explicit mode: explicit_challenges holds all num_rounds challenges, and the ones
 * already used must equal the transcript's. Where the first resumed round would take g(1)
 * from the recorded claim (a round of 2^12 pairs or more), it evaluates g(1) from the
 * tables and checks g(0) + g(1) against that claim on the device: tables other than the
 * ones the recorded rounds were proved on, or an altered claim, fail with SC_ERR_DEVICE
 * (device status 1) and leave the transcript unchanged. Synchronous, like sc_prove. */
int sc_prove_resume(sc_ctx* ctx, const sc_field* field, const sc_expr* expr,
                    const uint32_t* tables_dev, const uint32_t* explicit_challenges, int stop_round,
                    uint32_t* transcript, uint64_t words);

/* ---- Served proving -------------------------------------------------------------------
 * Replaces: nothing in the reference runs more than one proof at a time; its callers loop
 * over proofs (cuda/src/field_sumcheck.cu:1178-1336, src/zkduel/api.py:26-64).
 *
 * A server owns one GPU stream, a device memory pool and a worker thread. A request is the
 * call (expression, num_rounds, table kinds, seed, challenge mode): its tables are
 * generated on the device from the seed when it is admitted and stay resident, with its
 * fold buffers and transcript state, until it completes. Requests are admitted in arrival
 * order while the sum of admitted footprints (tables + fold buffers + partials + state)
 * stays within hbm_budget_bytes and fewer than max_inflight are in flight.
 *
 * SC_SERVE_CONTINUOUS: continuous batching. A request whose round 0 is larger than one wave
 *   of the GPU runs whole on a low-priority stream (one launch per round, one block per
 *   tile); the others are batched in ticks on high-priority streams, so they overtake the
 *   large proofs on the device. Every tick is one launch per degree class of
 *   the batched round kernel over (request, tile) items of the in-flight requests: each
 *   request whose current round has at most one wave of tiles left runs all of them, and
 *   the larger rounds share `chunk_items` tiles per tick, oldest request first (it gets one
 *   wave at least), advancing over several ticks. Requests join at the next tick after
 *   admission and leave after their last round, so arrivals overlap on the device with
 *   work already running.
 * SC_SERVE_FIFO_PLAIN: the baseline; one request at a time, in arrival order, each proved
 *   by the plain path (sc_prove) after its tables are generated.
 * Results are bit-identical to sc_prove on sc_tables_generate's tables for the same seed.
 * Times are seconds on the host's steady clock since sc_server_create. */
typedef struct sc_server sc_server;

#define SC_SERVE_CONTINUOUS 0
#define SC_SERVE_FIFO_PLAIN 1

typedef struct sc_server_stats {
  uint64_t submitted, completed, failed, suspended;
  uint64_t ticks;              /* launches groups issued (continuous policy) */
  uint64_t items;              /* (request, tile) items issued */
  uint64_t peak_inflight;      /* most requests admitted at once */
  uint64_t peak_footprint;     /* most bytes admitted at once */
  uint64_t budget;             /* hbm_budget_bytes */
  double busy_s;               /* host-observed time with at least one request in flight */
  double alloc_s;              /* worker time in pool allocations (admission) */
  double wait_s;               /* worker time blocked on the GPU (tick ring full / draining) */
  double build_s;              /* worker time composing and issuing ticks */
} sc_server_stats;

/* threads: 0 = default; pairs_per_thread: 0 = 1 (a tile is threads x pairs_per_thread
 * pairs); chunk_items: tiles per tick for the larger rounds, 0 = two waves of the grid. */
int sc_server_create(int device, const sc_field* field, int policy, uint64_t hbm_budget_bytes,
                     int max_inflight, int max_tables, int threads, int pairs_per_thread,
                     int chunk_items, sc_server** out);
/* Maps `bytes` of device memory into the server's pool ahead of time (allocates and frees
 * them; the pool keeps freed memory), so admissions up to that much do not grow the pool
 * while requests run. Synchronous. */
int sc_server_reserve(sc_server* server, uint64_t bytes);
/* Footprint a request would be admitted with; SC_ERR_UNSUPPORTED beyond the budget. */
int sc_server_footprint(const sc_server* server, const sc_expr* expr, int num_rounds,
                        uint64_t* out_bytes);
/* Queues a request (thread-safe; returns at once). table_kinds: expr's num_vars entries
 * of SC_TABLE_*. The expression is copied. */
int sc_server_submit(sc_server* server, const sc_expr* expr, int num_rounds,
                     const int32_t* table_kinds, uint64_t seed, int challenge_mode,
                     uint64_t* out_id);
/* Waits until request `id` completed (SC_OK), failed (its error code), or timeout_ms
 * passed (SC_ERR_TIMEOUT). timeout_ms < 0 waits without limit. */
int sc_server_wait(sc_server* server, uint64_t id, int timeout_ms);
/* Waits until every submitted request completed or failed. */
int sc_server_drain(sc_server* server, int timeout_ms);
/* Outputs of a completed request, laid out as sc_prove's; SC_ERR_PENDING before that. */
int sc_server_result(sc_server* server, uint64_t id, uint32_t* out_round_polys,
                     uint32_t* out_challenges, uint32_t* out_finals, uint32_t* out_claim0,
                     uint64_t* out_checksum);
/* Submit, admission and completion times of a request (completion: when the server saw
 * its last round and result copy finish). */
int sc_server_times(sc_server* server, uint64_t id, double* out_submit_s, double* out_admit_s,
                    double* out_done_s);
/* Forgets a completed request (its result is no longer readable). */
int sc_server_release(sc_server* server, uint64_t id);
/* Suspends request `id` (0: every request not finished) at its next round boundary: its
 * device memory goes back to the pool and its transcript is kept; sc_server_wait then
 * returns SC_SUSPENDED. Queued requests are suspended where they stand (rounds done as
 * submitted). Requests that finish first, and large requests already issued whole on
 * the lane, complete normally. Thread-safe; returns at once. */
int sc_server_suspend(sc_server* server, uint64_t id);
/* Transcript of a suspended request (sc_transcript_words words; carries the tag of its
 * seeded tables). */
int sc_server_transcript(sc_server* server, uint64_t id, uint32_t* transcript, uint64_t words);
/* Queues a request that continues the transcript's proof: the same expression, rounds,
 * table kinds and seed as the transcript's tables (the tag is checked), its challenge mode
 * (SHA3 or fixed). The tables are generated from the seed again and folded to the
 * transcript's round at admission; results are bit-identical to the uninterrupted proof. */
int sc_server_submit_resume(sc_server* server, const sc_expr* expr, const int32_t* table_kinds,
                            uint64_t seed, const uint32_t* transcript, uint64_t words,
                            uint64_t* out_id);
int sc_server_stats_get(sc_server* server, sc_server_stats* out);
/* Stops accepting requests, finishes the queued ones, joins the worker, frees everything. */
int sc_server_destroy(sc_server* server);

#ifdef __cplusplus
}
#endif

#endif /* SUMCHECK_B200_H */
