// libsumcheck_b200: the C ABI declared in include/sumcheck_b200.h.
//
// Host side of the prover: field and expression set-up, the scratch-owning context,
// table generation and the per-proof launch sequence. The reference drives its CUDA
// kernels from a CLI loop with a blocking device-to-host copy per interpolation point
// (cuda/src/field_sumcheck.cu:1012-1088); here a proof is num_rounds launches of one
// fused round kernel on the caller's stream and a single copy of the results at the end.
#include "host_common.h"
#include "prover_pp.cuh"

using namespace sc;
using namespace sc_host;

namespace {

// Rounds with at least this many pairs derive g(1) from the claim instead of evaluating
// point 1; the previous round then interpolates g_{j-1}(r_{j-1}) in its finalisation, a
// latency only worth paying when the round is large.
constexpr uint64_t kSkip1MinPairs = uint64_t{1} << 12;

inline bool round_skip1(int n, int j) { return j >= 1 && (uint64_t{1} << (n - j - 1)) >= kSkip1MinPairs; }

// Tail launch: from the first round with at most a few pairs a thread of the batched kernel's
// block (tail_round), that one block proves the rest of the proof (batch_round_kernel's tail rounds: no
// grid-wide partials and no launch per round). Generic expressions only: the batched kernel
// has no compile-time shapes, and the shape kernels' small rounds beat its generic evaluator.
// Measured on B200 (median of 10 proofs): a b over 2^32 - 5, n = 16, 0.254 -> 0.228 ms,
// n = 8 0.147 -> 0.110 ms; a degree-3 expression over 2^127 - 1, n = 8..20, 1.09-1.36x;
// with the zerocheck and g(abc + de) shapes, 0.91-1.0x (so those keep a launch per round).
#ifndef SC_PLAIN_TAILS
#define SC_PLAIN_TAILS 1
#endif
constexpr bool kPlainTails = SC_PLAIN_TAILS != 0;

struct TailDesc {
  BatchRound r;
  ExprDev e;
};

int tail_shape(sc_ctx* ctx, int L, int kind, int dclass, int tables, int* threads, size_t* smem) {
  for (const TailShape& t : ctx->tail_shapes)
    if (t.L == L && t.kind == kind && t.dclass == dclass && t.tables == tables) {
      *threads = t.threads;
      *smem = t.smem;
      return SC_OK;
    }
  int grid = 0;
  int rc = batch_kernel_setup(L, kind, dclass, tables, 0, ctx->sm_count, threads, &grid, smem);
  if (rc) return rc;
  ctx->tail_shapes.push_back(TailShape{L, kind, dclass, tables, *threads, *smem});
  return SC_OK;
}

// The round the tail launch starts at (stop: none), for a proof run up to round stop: the
// first with at most a few pairs a thread of the batched kernel's block.
int tail_round(sc_ctx* ctx, int L, int kind, int dclass, int tables, int shape, int n, int first, int stop,
               int* out_round, int* threads, size_t* smem) {
  *out_round = stop;
  if (!kPlainTails || stop != n || shape != kShapeGeneric) return SC_OK;
  int rc = tail_shape(ctx, L, kind, dclass, tables, threads, smem);
  if (rc) return rc;
  // pairs a thread at the tail's first round: measured on B200 (1, 2 or 4), 4 was best for
  // a b over 2^32 - 5 (n = 16: 0.233 -> 0.224 ms), 1-2 for 4 and 8 limbs (4 was 3-7% slower)
  const uint64_t per_thread = L == 1 ? 4 : (L <= 4 ? 2 : 1);
  for (int j = first; j < n - 1; ++j)
    if (((uint64_t{1} << n) >> (j + 1)) <= static_cast<uint64_t>(*threads) * per_thread) {
      *out_round = j;
      break;
    }
  return SC_OK;
}

template <int L, int K, int DMAX>
struct ProveRun {
  // Rounds [first, stop) of the proof. state_io (host, state words; NULL for a whole proof
  // from round 0): the state after round first - 1 in, the state after round stop - 1 out.
  static int run(sc_ctx* ctx, const sc_field* f, const sc_expr* ex, int n, const uint32_t* tables, int mode,
                 const uint32_t* explicit_ch, uint32_t* out_polys, uint32_t* out_ch, uint32_t* out_finals,
                 uint32_t* out_claim0, uint64_t* out_checksum, int first, int stop, uint32_t* state_io) {
    const int K_ = ex->num_vars;
    const uint64_t N = uint64_t{1} << n;
    // scratch
    const size_t fold_a_words = n >= 2 ? static_cast<size_t>(K_) * L * (N / 2) : 0;
    const size_t fold_b_words = n >= 3 ? static_cast<size_t>(K_) * L * (N / 4) : 0;
    int rc;
    if ((rc = ensure(ctx, ctx->fold_a, fold_a_words * 4))) return rc;
    if ((rc = ensure(ctx, ctx->fold_b, fold_b_words * 4))) return rc;
    const StateOffsets so = state_offsets(n, K_, L);
    if ((rc = ensure(ctx, ctx->state, so.total_words * 4))) return rc;

    ExprDev E;
    build_expr_dev<L>(*ex, *f, E);
    // the kernel: a compile-time shape when the expression has one, else the generic evaluator
    using Kern = void (*)(const RoundArgs, const ExprDev, const FieldParams<L, K>);
    Kern kern = round_kernel<L, K, DMAX>;
    int shape = kShapeGeneric;
    if constexpr (DMAX == 4) {
      if (E.shape == kShapeZerocheck) kern = round_kernel<L, K, 4, kShapeZerocheck>;
      if (E.shape == kShapeAbcg) kern = round_kernel<L, K, 4, kShapeAbcg>;
      shape = E.shape;
    }
    int threads = kernel_threads(L);
    size_t smem;
    if (use_point_parallel(L) && shape == kShapeGeneric) {
      kern = round_kernel_pp<L, K>;
      threads = kPointParallelThreads;
      smem = static_cast<size_t>(pp_smem_words(threads, K_, L)) * 4;
      SC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem));
    } else if (shape == kShapeGeneric) {
      const int per_thread = round_smem_words_per_thread(K_, L) * 4;
      while (threads > 32 && threads * per_thread > kMaxDynSmem) threads -= 32;
      smem = static_cast<size_t>(threads) * per_thread;
    } else {
      smem = shape_round_smem_bytes(L, K, shape, threads);  // block_reduce scratch (+ the pair stage)
    }
    int blocks_per_sm = 0;
    SC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, threads, smem));
    if (blocks_per_sm < 1) return fail(SC_ERR_UNSUPPORTED, "round kernel does not fit on an SM (K=%d, L=%d)", K_, L);
    const uint64_t grid_max = static_cast<uint64_t>(blocks_per_sm) * ctx->sm_count;
    if ((rc = ensure(ctx, ctx->partials, grid_max * kMaxPoints * L * 4))) return rc;

    FieldParams<L, K> F;
    for (int l = 0; l < L; ++l) F.p[l] = f->hf.p[l];
    F.np = f->hf.np;

    uint32_t* st = static_cast<uint32_t*>(ctx->state.p);
    if (state_io)
      SC_CUDA(cudaMemcpyAsync(st, state_io, so.total_words * 4, cudaMemcpyHostToDevice, ctx->stream));
    else
      SC_CUDA(cudaMemsetAsync(st, 0, so.total_words * 4, ctx->stream));
    if (mode == SC_CHALLENGE_EXPLICIT)
      SC_CUDA(cudaMemcpyAsync(st + so.chals, explicit_ch, static_cast<size_t>(n) * L * 4, cudaMemcpyHostToDevice,
                              ctx->stream));

    RoundArgs A;
    std::memset(&A, 0, sizeof(A));
    A.num_rounds = n;
    A.mode = mode;
    A.partials = static_cast<uint32_t*>(ctx->partials.p);
    A.fc = f->dev;
    A.st.counter = st + so.counter;
    A.st.status = st + so.status;
    A.st.checksum = reinterpret_cast<uint64_t*>(st + so.checksum);
    A.st.polys = st + so.polys;
    A.st.chals = st + so.chals;
    A.st.finals = st + so.finals;
    A.st.claim0 = st + so.claim0;
    A.st.claim = st + so.claim;

    // T_{first-1} (or T_0), refolded from T_0 with the recorded challenges when resuming
    if ((rc = resume_folds(f, n, K_, tables, static_cast<uint32_t*>(ctx->fold_a.p), static_cast<uint32_t*>(ctx->fold_b.p),
                           st + so.chals, first, ctx->sm_count, ctx->stream)))
      return rc;
    const uint32_t* prev = first <= 1 ? tables : static_cast<const uint32_t*>(((first - 1) & 1) ? ctx->fold_a.p : ctx->fold_b.p);
    int tail_j = stop, tail_threads = 0;
    size_t tail_smem = 0;
    if ((rc = tail_round(ctx, L, K, DMAX, K_, shape, n, first, stop, &tail_j, &tail_threads, &tail_smem))) return rc;
    for (int j = first; j < stop; ++j) {
      A.round = j;
      A.pairs = N >> (j + 1);
      A.skip1 = round_skip1(n, j) ? 1 : 0;
      A.want_claim = (j + 1 < n && round_skip1(n, j + 1)) ? 1 : 0;
      // The first round of a resumed segment whose recorded claim is defined (the round
      // would take g(1) from it) evaluates g(1) from the tables instead and checks
      // g(0) + g(1) against that claim: tables other than the ones the recorded rounds were
      // proved on, or an altered claim, fail with kStatusClaim. Equal values either way, so
      // the proof is unchanged.
      A.check_claim = (state_io && j == first && A.skip1) ? 1 : 0;
      if (A.check_claim) A.skip1 = 0;
      if (j == 0) {
        A.fold = 0;
        A.src = tables;
        A.dst = nullptr;
        A.src_len = N;
      } else {
        A.fold = 1;
        A.src = prev;
        A.src_len = N >> (j - 1);
        A.dst = static_cast<uint32_t*>((j & 1) ? ctx->fold_a.p : ctx->fold_b.p);
        prev = A.dst;
      }
      if (j == tail_j) {  // this round and every later one, in one block
        if ((rc = ensure(ctx, ctx->tail, sizeof(TailDesc)))) return rc;
        if (!ctx->tail_host) SC_CUDA(cudaMallocHost(&ctx->tail_host, sizeof(TailDesc)));
        if (!ctx->tail_copied) SC_CUDA(cudaEventCreateWithFlags(&ctx->tail_copied, cudaEventDisableTiming));
        // the staging's previous copy has landed (a proof ends with a stream synchronisation,
        // unless it failed part way)
        SC_CUDA(cudaEventSynchronize(ctx->tail_copied));
        TailDesc& desc = *static_cast<TailDesc*>(ctx->tail_host);
        std::memset(&desc, 0, sizeof(desc));
        TailDesc* dev = static_cast<TailDesc*>(ctx->tail.p);
        desc.r.args = A;
        desc.r.expr = &dev->e;
        desc.r.partials = A.partials;
        desc.r.num_items = 1;
        desc.r.round_items = 1;
        desc.r.tail_rounds = n - 1 - j;
        desc.r.skip1_min_pairs = static_cast<uint32_t>(kSkip1MinPairs);
        desc.r.fold_a = static_cast<uint32_t*>(ctx->fold_a.p);
        desc.r.fold_b = static_cast<uint32_t*>(ctx->fold_b.p);
        desc.e = E;
        SC_CUDA(cudaMemcpyAsync(dev, &desc, sizeof(desc), cudaMemcpyHostToDevice, ctx->stream));
        SC_CUDA(cudaEventRecord(ctx->tail_copied, ctx->stream));
        BatchTickArgs T;
        T.rounds = &dev->r;
        T.items = nullptr;
        T.num_items = 1;
        T.pad = 0;
        T.head = nullptr;
        T.tile = A.pairs;
        cudaEvent_t ev;
        if ((rc = timing_begin(ctx, &ev))) return rc;
        if ((rc = batch_kernel_launch(L, K, DMAX, f, 1, tail_threads, tail_smem, ctx->stream, T))) return rc;
        if ((rc = timing_end(ctx))) return rc;
        break;
      }
      uint64_t per_block = static_cast<uint64_t>(threads);
      if (use_point_parallel(L) && shape == kShapeGeneric) {  // pairs a block holds: one per lane group
        const int npts = ex->degree + 1 - (A.skip1 ? 1 : 0);
        const int G = npts <= 2 ? 2 : (npts <= 4 ? 4 : 8);
        per_block = static_cast<uint64_t>(threads / G);
      }
      const uint64_t want = (A.pairs + per_block - 1) / per_block;
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(want, grid_max));
      cudaEvent_t ev;
      if ((rc = timing_begin(ctx, &ev))) return rc;
      kern<<<grid, threads, smem, ctx->stream>>>(A, E, F);
      SC_CUDA(cudaGetLastError());
      if ((rc = timing_end(ctx))) return rc;
    }
    return finish(ctx, ex, n, stop, st, so, out_polys, out_ch, out_finals, out_claim0, out_checksum, state_io);
  }

  // One copy of the state to pinned memory, then the caller's arrays (outputs only when the
  // proof is complete) and the state words.
  static int finish(sc_ctx* ctx, const sc_expr* ex, int n, int stop, const uint32_t* st, const StateOffsets& so,
                    uint32_t* out_polys, uint32_t* out_ch, uint32_t* out_finals, uint32_t* out_claim0,
                    uint64_t* out_checksum, uint32_t* state_io) {
    const int d = ex->degree, K_ = ex->num_vars;
    int rc;
    if (ctx->host_state_bytes < so.total_words * 4) {
      if (ctx->host_state) cudaFreeHost(ctx->host_state);
      ctx->host_state = nullptr;
      ctx->host_state_bytes = 0;
      SC_CUDA(cudaMallocHost(&ctx->host_state, so.total_words * 4));
      ctx->host_state_bytes = so.total_words * 4;
    }
    SC_CUDA(cudaMemcpyAsync(ctx->host_state, st, so.total_words * 4, cudaMemcpyDeviceToHost, ctx->stream));
    SC_CUDA(cudaStreamSynchronize(ctx->stream));
    if ((rc = timing_collect(ctx))) return rc;
    const uint32_t* hs = ctx->host_state;
    if (hs[so.status]) return fail(SC_ERR_DEVICE, "device status %u", hs[so.status]);
    if (state_io) std::memcpy(state_io, hs, so.total_words * 4);
    if (stop < n) return SC_OK;
    if (out_polys)
      for (int j = 0; j < n; ++j)
        std::memcpy(out_polys + static_cast<size_t>(j) * (d + 1) * L, hs + so.polys + static_cast<size_t>(j) * kMaxPoints * L,
                    static_cast<size_t>(d + 1) * L * 4);
    if (out_ch) std::memcpy(out_ch, hs + so.chals, static_cast<size_t>(n) * L * 4);
    if (out_finals) std::memcpy(out_finals, hs + so.finals, static_cast<size_t>(1 + K_) * L * 4);
    if (out_claim0) std::memcpy(out_claim0, hs + so.claim0, L * 4);
    if (out_checksum) std::memcpy(out_checksum, hs + so.checksum, 8);
    return SC_OK;
  }
};

template <int L, int K>
int fold_prefix(const sc_field* f, int n, int num_tables, const uint32_t* tables, uint32_t* fold_a, uint32_t* fold_b,
                const uint32_t* chals_dev, int j, int sm_count, cudaStream_t stream) {
  FieldParams<L, K> F;
  for (int l = 0; l < L; ++l) F.p[l] = f->hf.p[l];
  F.np = f->hf.np;
  const uint64_t N = uint64_t{1} << n;
  const uint32_t* src = tables;
  for (int i = 1; i < j; ++i) {
    uint32_t* dst = (i & 1) ? fold_a : fold_b;
    const uint64_t src_len = N >> (i - 1);
    const uint64_t total = (src_len >> 2) * static_cast<uint64_t>(num_tables);
    const unsigned grid = static_cast<unsigned>(
        std::max<uint64_t>(1, std::min<uint64_t>((total + 255) / 256, static_cast<uint64_t>(sm_count) * 8)));
    fold_kernel<L, K><<<grid, 256, 0, stream>>>(src, dst, src_len, num_tables, chals_dev + static_cast<size_t>(i - 1) * L, F);
    SC_CUDA(cudaGetLastError());
    src = dst;
  }
  return SC_OK;
}

template <int L>
int generate_impl(sc_ctx* ctx, const sc_field* f, int num_tables, int n, const int32_t* kinds,
                  uint64_t seed, uint32_t* tables) {
  TableGenArgs G;
  std::memset(&G, 0, sizeof(G));
  G.num_tables = num_tables;
  G.entries = uint64_t{1} << n;
  G.seed = seed;
  for (int k = 0; k < num_tables; ++k) G.kinds[k] = kinds[k];
  const HostField& hf = f->hf;
  int bits = 0;
  for (int l = L - 1; l >= 0 && !bits; --l)
    if (hf.p[l]) bits = 32 * l + (32 - __builtin_clz(hf.p[l]));
  for (int l = 0; l < L; ++l) {
    const int lo = 32 * l;
    G.mask[l] = bits >= lo + 32 ? 0xFFFFFFFFu : (bits <= lo ? 0u : ((1u << (bits - lo)) - 1u));
  }
  bool fits64 = true;
  for (int l = 2; l < L; ++l) fits64 = fits64 && hf.p[l] == 0;
  G.p_u64 = fits64 ? (static_cast<uint64_t>(L > 1 ? hf.p[1] : 0) << 32) | hf.p[0] : 0;
  for (int l = 0; l < L; ++l) G.r2[l] = f->consts.r2[l];
  FieldParams<L> F;
  for (int l = 0; l < L; ++l) F.p[l] = hf.p[l];
  F.np = hf.np;
  const uint64_t total = G.entries * num_tables;
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((total + 255) / 256, uint64_t{1} << 30));
  generate_tables_kernel<L><<<grid, 256, 0, ctx->stream>>>(G, F, tables);
  SC_CUDA(cudaGetLastError());
  return SC_OK;
}

template <int L>
int convert_impl(sc_ctx* ctx, const sc_field* f, uint32_t* tables, uint64_t entries, int num_tables, bool to_mont) {
  FieldParams<L> F;
  for (int l = 0; l < L; ++l) F.p[l] = f->hf.p[l];
  F.np = f->hf.np;
  Fe<L> factor;
  for (int l = 0; l < L; ++l) factor.w[l] = to_mont ? f->consts.r2[l] : (l == 0 ? 1u : 0u);
  const uint64_t total = entries * num_tables;
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((total + 255) / 256, uint64_t{1} << 30));
  convert_tables_kernel<L><<<grid, 256, 0, ctx->stream>>>(tables, entries, num_tables, factor, F);
  SC_CUDA(cudaGetLastError());
  return SC_OK;
}

template <int L>
int apply_impl(sc_ctx* ctx, const sc_field* f, int op, const uint32_t* a, const uint32_t* b, uint32_t* out,
               uint64_t count) {
  FieldParams<L> F;
  for (int l = 0; l < L; ++l) F.p[l] = f->hf.p[l];
  F.np = f->hf.np;
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((count + 255) / 256, uint64_t{1} << 30));
  field_apply_kernel<L><<<grid, 256, 0, ctx->stream>>>(op, a, b, out, count, F);
  SC_CUDA(cudaGetLastError());
  return SC_OK;
}

}  // namespace

extern "C" {

int sc_version(void) { return 100; }

const char* sc_last_error(void) { return g_err.c_str(); }

int sc_ctx_create(int device, void* stream, sc_ctx** out) {
  if (!out) return fail(SC_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int count = 0;
  SC_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(SC_ERR_INVALID, "device %d out of range (%d devices)", device, count);
  SC_CUDA(cudaSetDevice(device));
  sc_ctx* c = new (std::nothrow) sc_ctx();
  if (!c) return fail(SC_ERR_NOMEM, "host allocation failed");
  c->device = device;
  c->stream = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    delete c;
    return fail(SC_ERR_CUDA, "cudaDeviceGetAttribute: %s", cudaGetErrorString(e));
  }
  int rc;
  if ((rc = for_each_instance<SetRoundAttrs>())) {
    delete c;
    return rc;
  }
  *out = c;
  return SC_OK;
}

int sc_ctx_destroy(sc_ctx* ctx) {
  if (!ctx) return SC_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (DevBuf* b : {&ctx->fold_a, &ctx->fold_b, &ctx->partials, &ctx->state, &ctx->tail})
    if (b->p) cudaFree(b->p);
  for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
  if (ctx->host_state) cudaFreeHost(ctx->host_state);
  if (ctx->tail_host) cudaFreeHost(ctx->tail_host);
  if (ctx->tail_copied) cudaEventDestroy(ctx->tail_copied);
  delete ctx;
  return SC_OK;
}

int sc_ctx_synchronize(sc_ctx* ctx) {
  if (!ctx) return fail(SC_ERR_INVALID, "ctx is NULL");
  SC_CUDA(cudaStreamSynchronize(ctx->stream));
  return timing_collect(ctx);
}

int sc_ctx_set_timing(sc_ctx* ctx, int enable) {
  if (!ctx) return fail(SC_ERR_INVALID, "ctx is NULL");
  SC_CUDA(cudaStreamSynchronize(ctx->stream));
  int rc = timing_collect(ctx);
  ctx->timing = enable != 0;
  ctx->launch_ms.clear();
  return rc;
}

int sc_ctx_launch_times(sc_ctx* ctx, float* out_ms, int capacity, int* count) {
  if (!ctx || !count) return fail(SC_ERR_INVALID, "NULL argument");
  const int n = static_cast<int>(ctx->launch_ms.size());
  *count = n;
  const int take = out_ms ? std::min(n, std::max(capacity, 0)) : 0;
  for (int i = 0; i < take; ++i) out_ms[i] = ctx->launch_ms[i];
  ctx->launch_ms.erase(ctx->launch_ms.begin(), ctx->launch_ms.begin() + take);
  return SC_OK;
}

int sc_field_init(int limbs, const uint32_t* modulus, uint32_t nprime, sc_field** out) {
  if (!out || !modulus) return fail(SC_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (limbs != 1 && limbs != 2 && limbs != 4 && limbs != 8)
    return fail(SC_ERR_UNSUPPORTED, "limbs must be 1, 2, 4 or 8, got %d", limbs);
  sc_field* f = new (std::nothrow) sc_field();
  if (!f) return fail(SC_ERR_NOMEM, "host allocation failed");
  HostField& hf = f->hf;
  hf.L = limbs;
  std::memcpy(hf.p, modulus, 4 * limbs);
  hf.np = nprime;
  bool big = false;
  for (int l = 1; l < limbs; ++l) big = big || hf.p[l];
  if (!(hf.p[0] & 1u) || (!big && hf.p[0] < 3)) {
    delete f;
    return fail(SC_ERR_UNSAFE_MODULUS, "Montgomery arithmetic needs an odd modulus > 2");
  }
  uint32_t inv = 1;  // p^-1 mod 2^32 by Newton iteration
  for (int i = 0; i < 5; ++i) inv *= 2u - hf.p[0] * inv;
  if (nprime != 0u - inv) {
    delete f;
    return fail(SC_ERR_UNSAFE_MODULUS, "nprime %#x != -p^-1 mod 2^32 = %#x", nprime, 0u - inv);
  }
  if (!cios_bound_holds(hf)) {
    delete f;
    return fail(SC_ERR_UNSAFE_MODULUS,
                "the device Montgomery routine does not support this modulus; it is valid only "
                "when (2p-1) + (p-1)(2^32-1) < 2^(32(L+1))");
  }
  FieldConsts& C = f->consts;
  std::memset(&C, 0, sizeof(C));
  std::memcpy(C.p, hf.p, 4 * limbs);
  C.np = nprime;
  C.limbs = limbs;
  C.p_small = big ? 0u : hf.p[0];
  // R mod p, R^2 mod p, R^2 2^(32 i) mod p by doubling from 1
  uint32_t x[8] = {0};
  x[0] = 1;
  for (int i = 0; i < 32 * limbs; ++i) hf.dbl(x, x);
  std::memcpy(C.one, x, 4 * limbs);
  for (int i = 0; i < 32 * limbs; ++i) hf.dbl(x, x);
  std::memcpy(C.r2, x, 4 * limbs);
  for (int w = 0; w < 8; ++w) {
    std::memcpy(C.kdig[w], x, 4 * limbs);
    for (int i = 0; i < 32; ++i) hf.dbl(x, x);
  }
  for (int t = 0; t < kMaxPoints; ++t) mont_small(hf, C.r2, static_cast<uint64_t>(t), C.pts[t]);
  // Lagrange weights 1 / prod_{s != t} (t - s) (Fermat inverse; verified, p must be prime)
  uint32_t pm2[8];
  std::memcpy(pm2, hf.p, 32);
  pm2[0] -= 2;  // p odd and > 2: no borrow unless p[0] < 2, handled below
  if (hf.p[0] < 2) {
    uint32_t two[8] = {2};
    hf.sub_raw(hf.p, two, pm2);
  }
  for (int d = 0; d < kMaxPoints; ++d)
    for (int t = 0; t <= d; ++t) {
      int64_t den = 1;
      for (int s = 0; s <= d; ++s)
        if (s != t) den *= (t - s);
      uint32_t dm[8];
      mont_small(hf, C.r2, static_cast<uint64_t>(den < 0 ? -den : den), dm);
      if (den < 0) hf.neg(dm, dm);
      uint32_t inv_m[8], chk[8];
      mont_pow(hf, dm, pm2, C.one, inv_m);
      hf.mul(inv_m, dm, chk);
      if (std::memcmp(chk, C.one, 4 * limbs) != 0) f->has_inverses = false;
      std::memcpy(C.lag[d][t], inv_m, 4 * limbs);
    }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaMalloc(&f->dev, sizeof(FieldConsts));
  if (e == cudaSuccess) e = cudaMemcpy(f->dev, &C, sizeof(FieldConsts), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (f->dev) cudaFree(f->dev);
    delete f;
    return fail(SC_ERR_CUDA, "field constants upload: %s", cudaGetErrorString(e));
  }
  f->device = dev;
  *out = f;
  return SC_OK;
}

int sc_field_destroy(sc_field* field) {
  if (!field) return SC_OK;
  if (field->dev) cudaFree(field->dev);
  delete field;
  return SC_OK;
}

int sc_expr_compile(int num_vars, int num_terms, const int64_t* coeffs, const uint32_t* coeff_limbs,
                    const int32_t* term_lens, const int32_t* term_offsets, const int32_t* flat,
                    sc_expr** out) {
  if (!out || !term_lens || !term_offsets || !flat || (!coeffs && !coeff_limbs))
    return fail(SC_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (num_vars < 1 || num_vars > kMaxVars) return fail(SC_ERR_UNSUPPORTED, "num_vars %d outside 1..%d", num_vars, kMaxVars);
  if (num_terms < 1 || num_terms > kMaxTerms) return fail(SC_ERR_UNSUPPORTED, "num_terms %d outside 1..%d", num_terms, kMaxTerms);
  sc_expr* ex = new (std::nothrow) sc_expr();
  if (!ex) return fail(SC_ERR_NOMEM, "host allocation failed");
  ex->num_vars = num_vars;
  ex->num_terms = num_terms;
  int total = 0, degree = 0;
  for (int i = 0; i < num_terms; ++i) {
    if (term_lens[i] < 1 || term_offsets[i] != total) {
      delete ex;
      return fail(SC_ERR_INVALID, "term %d: length %d / offset %d (expected offset %d)", i, term_lens[i], term_offsets[i], total);
    }
    total += term_lens[i];
    degree = std::max(degree, static_cast<int>(term_lens[i]));
  }
  if (total > kMaxFlat) {
    delete ex;
    return fail(SC_ERR_UNSUPPORTED, "%d factors exceed %d", total, kMaxFlat);
  }
  if (degree > kMaxPoints - 1) {
    delete ex;
    return fail(SC_ERR_UNSUPPORTED, "degree %d exceeds %d", degree, kMaxPoints - 1);
  }
  for (int i = 0; i < total; ++i)
    if (flat[i] < 0 || flat[i] >= num_vars) {
      delete ex;
      return fail(SC_ERR_INVALID, "factor %d refers to table %d of %d", i, flat[i], num_vars);
    }
  ex->degree = degree;
  ex->coeffs.assign(num_terms, 0);
  if (coeffs) ex->coeffs.assign(coeffs, coeffs + num_terms);
  if (coeff_limbs) ex->coeff_limbs.assign(coeff_limbs, coeff_limbs + 8 * num_terms);
  ex->lens.assign(term_lens, term_lens + num_terms);
  ex->offs.assign(term_offsets, term_offsets + num_terms);
  ex->flat.assign(flat, flat + total);
  *out = ex;
  return SC_OK;
}

int sc_expr_destroy(sc_expr* expr) {
  delete expr;
  return SC_OK;
}

int sc_expr_degree(const sc_expr* expr) { return expr ? expr->degree : -1; }
int sc_expr_num_vars(const sc_expr* expr) { return expr ? expr->num_vars : -1; }

int sc_tables_generate(sc_ctx* ctx, const sc_field* field, int num_tables, int num_rounds,
                       const int32_t* kinds, uint64_t seed, uint32_t* tables_dev) {
  if (!ctx || !field || !kinds || !tables_dev) return fail(SC_ERR_INVALID, "NULL argument");
  if (num_tables < 1 || num_tables > kMaxVars) return fail(SC_ERR_INVALID, "num_tables %d outside 1..%d", num_tables, kMaxVars);
  if (num_rounds < 1 || num_rounds > kMaxRounds) return fail(SC_ERR_INVALID, "num_rounds %d outside 1..%d", num_rounds, kMaxRounds);
  for (int k = 0; k < num_tables; ++k)
    if (kinds[k] < 0) return fail(SC_ERR_INVALID, "kinds[%d] = %d", k, kinds[k]);
  if (reinterpret_cast<uintptr_t>(tables_dev) % 16) return fail(SC_ERR_INVALID, "tables_dev must be 16-byte aligned");
  switch (field->hf.L) {
    case 1: return generate_impl<1>(ctx, field, num_tables, num_rounds, kinds, seed, tables_dev);
    case 2: return generate_impl<2>(ctx, field, num_tables, num_rounds, kinds, seed, tables_dev);
    case 4: return generate_impl<4>(ctx, field, num_tables, num_rounds, kinds, seed, tables_dev);
    default: return generate_impl<8>(ctx, field, num_tables, num_rounds, kinds, seed, tables_dev);
  }
}

static int convert(sc_ctx* ctx, const sc_field* field, uint32_t* tables, uint64_t entries, int num_tables, bool to_mont) {
  if (!ctx || !field || !tables) return fail(SC_ERR_INVALID, "NULL argument");
  if (num_tables < 1 || entries == 0) return fail(SC_ERR_INVALID, "empty table set");
  switch (field->hf.L) {
    case 1: return convert_impl<1>(ctx, field, tables, entries, num_tables, to_mont);
    case 2: return convert_impl<2>(ctx, field, tables, entries, num_tables, to_mont);
    case 4: return convert_impl<4>(ctx, field, tables, entries, num_tables, to_mont);
    default: return convert_impl<8>(ctx, field, tables, entries, num_tables, to_mont);
  }
}

int sc_tables_to_mont(sc_ctx* ctx, const sc_field* field, uint32_t* tables_dev, uint64_t entries, int num_tables) {
  return convert(ctx, field, tables_dev, entries, num_tables, true);
}

int sc_tables_from_mont(sc_ctx* ctx, const sc_field* field, uint32_t* tables_dev, uint64_t entries, int num_tables) {
  return convert(ctx, field, tables_dev, entries, num_tables, false);
}

int sc_field_apply(sc_ctx* ctx, const sc_field* field, int op, const uint32_t* a_dev, const uint32_t* b_dev,
                   uint32_t* out_dev, uint64_t count) {
  if (!ctx || !field || !a_dev || !b_dev || !out_dev) return fail(SC_ERR_INVALID, "NULL argument");
  if (op < 0 || op > 2) return fail(SC_ERR_INVALID, "unknown op %d", op);
  if (count == 0) return SC_OK;
  switch (field->hf.L) {
    case 1: return apply_impl<1>(ctx, field, op, a_dev, b_dev, out_dev, count);
    case 2: return apply_impl<2>(ctx, field, op, a_dev, b_dev, out_dev, count);
    case 4: return apply_impl<4>(ctx, field, op, a_dev, b_dev, out_dev, count);
    default: return apply_impl<8>(ctx, field, op, a_dev, b_dev, out_dev, count);
  }
}

int sc_calibrate_imad(sc_ctx* ctx, double* out_imad_per_s) {
  if (!ctx || !out_imad_per_s) return fail(SC_ERR_INVALID, "NULL argument");
  SC_CUDA(cudaSetDevice(ctx->device));
  uint32_t* sink = nullptr;
  SC_CUDA(cudaMalloc(&sink, 16));
  const int threads = 512, iters = 4096;
  const int blocks = ctx->sm_count * 4;
  cudaEvent_t e0, e1;
  SC_CUDA(cudaEventCreate(&e0));
  SC_CUDA(cudaEventCreate(&e1));
  imad_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(sink, 64, 1u);  // warm-up
  float best = 0.f;
  for (int rep = 0; rep < 3; ++rep) {
    SC_CUDA(cudaEventRecord(e0, ctx->stream));
    imad_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(sink, iters, 7u + rep);
    SC_CUDA(cudaEventRecord(e1, ctx->stream));
    SC_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (best == 0.f || ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  const double ops = static_cast<double>(blocks) * threads * iters * 8.0 * 2.0;
  *out_imad_per_s = ops / (best * 1e-3);
  return SC_OK;
}

int sc_prove(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int num_rounds,
             const uint32_t* tables_dev, int challenge_mode, const uint32_t* explicit_challenges,
             uint32_t* out_round_polys, uint32_t* out_challenges, uint32_t* out_finals,
             uint32_t* out_claim0, uint64_t* out_checksum) {
  if (!ctx || !field || !expr || !tables_dev) return fail(SC_ERR_INVALID, "NULL argument");
  if (num_rounds < 1 || num_rounds > kMaxRounds)
    return fail(SC_ERR_INVALID, "num_rounds %d outside 1..%d", num_rounds, kMaxRounds);
  if (challenge_mode < SC_CHALLENGE_SHA3 || challenge_mode > SC_CHALLENGE_EXPLICIT)
    return fail(SC_ERR_INVALID, "unknown challenge mode %d", challenge_mode);
  if (challenge_mode == SC_CHALLENGE_EXPLICIT && !explicit_challenges)
    return fail(SC_ERR_INVALID, "explicit challenge mode needs explicit_challenges");
  if (reinterpret_cast<uintptr_t>(tables_dev) % 16) return fail(SC_ERR_INVALID, "tables_dev must be 16-byte aligned");
  if (field->device != ctx->device) return fail(SC_ERR_INVALID, "field was set up on device %d, context is on %d", field->device, ctx->device);
  SC_CUDA(cudaSetDevice(ctx->device));
  return dispatch<ProveRun>(field->hf.L, field_kind(field->hf.p, field->hf.L), degree_class(expr->degree), ctx, field,
                            expr, num_rounds, tables_dev, challenge_mode, explicit_challenges, out_round_polys,
                            out_challenges, out_finals, out_claim0, out_checksum, 0, num_rounds, nullptr);
}

}  // extern "C"

namespace sc_host {

int resume_folds(const sc_field* f, int n, int num_tables, const uint32_t* tables, uint32_t* fold_a, uint32_t* fold_b,
                 const uint32_t* chals_dev, int j, int sm_count, cudaStream_t stream) {
  if (j <= 1) return SC_OK;
  if (j > n - 1) return fail(SC_ERR_INVALID, "resume at round %d of %d", j, n);
  const int L = f->hf.L;
  switch (L) {
    case 1: return fold_prefix<1, kFieldGeneric>(f, n, num_tables, tables, fold_a, fold_b, chals_dev, j, sm_count, stream);
    case 2:
      return field_kind(f->hf.p, L) == kFieldGoldilocks
                 ? fold_prefix<2, kFieldGoldilocks>(f, n, num_tables, tables, fold_a, fold_b, chals_dev, j, sm_count, stream)
                 : fold_prefix<2, kFieldGeneric>(f, n, num_tables, tables, fold_a, fold_b, chals_dev, j, sm_count, stream);
    case 4:
      return field_kind(f->hf.p, L) == kFieldMersenne127
                 ? fold_prefix<4, kFieldMersenne127>(f, n, num_tables, tables, fold_a, fold_b, chals_dev, j, sm_count, stream)
                 : fold_prefix<4, kFieldGeneric>(f, n, num_tables, tables, fold_a, fold_b, chals_dev, j, sm_count, stream);
    default: return fold_prefix<8, kFieldGeneric>(f, n, num_tables, tables, fold_a, fold_b, chals_dev, j, sm_count, stream);
  }
}

int prove_segment(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int n, const uint32_t* tables, int mode,
                  const uint32_t* explicit_ch, int first, int stop, uint32_t* state_io) {
  if (first < 0 || stop <= first || stop > n) return fail(SC_ERR_INVALID, "rounds [%d, %d) of %d", first, stop, n);
  SC_CUDA(cudaSetDevice(ctx->device));
  return dispatch<ProveRun>(field->hf.L, field_kind(field->hf.p, field->hf.L), degree_class(expr->degree), ctx, field,
                            expr, n, tables, mode, explicit_ch, nullptr, nullptr, nullptr, nullptr, nullptr, first, stop,
                            state_io);
}

}  // namespace sc_host

extern "C" {

int sc_prove_launches(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int num_rounds, int* out_launches,
                      int* out_tail_round) {
  if (!ctx || !field || !expr) return fail(SC_ERR_INVALID, "NULL argument");
  if (num_rounds < 1 || num_rounds > kMaxRounds)
    return fail(SC_ERR_INVALID, "num_rounds %d outside 1..%d", num_rounds, kMaxRounds);
  SC_CUDA(cudaSetDevice(ctx->device));
  int tail = num_rounds, threads = 0;
  size_t smem = 0;
  uint8_t role[16];
  const int dclass = degree_class(expr->degree);
  const int shape = dclass == 4 ? match_shape(*expr, role) : kShapeGeneric;
  const int rc = tail_round(ctx, field->hf.L, field_kind(field->hf.p, field->hf.L), dclass, expr->num_vars, shape,
                            num_rounds, 0, num_rounds, &tail, &threads, &smem);
  if (rc) return rc;
  if (out_launches) *out_launches = tail < num_rounds ? tail + 1 : num_rounds;
  if (out_tail_round) *out_tail_round = tail;
  return SC_OK;
}

int sc_transcript_words(const sc_field* field, const sc_expr* expr, int num_rounds, uint64_t* out_words) {
  if (!field || !expr || !out_words) return fail(SC_ERR_INVALID, "NULL argument");
  if (num_rounds < 1 || num_rounds > kMaxRounds)
    return fail(SC_ERR_INVALID, "num_rounds %d outside 1..%d", num_rounds, kMaxRounds);
  *out_words = transcript_words(num_rounds, expr->num_vars, field->hf.L);
  return SC_OK;
}

int sc_transcript_init(const sc_field* field, const sc_expr* expr, int num_rounds, int challenge_mode,
                       uint64_t tables_tag, uint32_t* transcript, uint64_t words) {
  uint64_t need = 0;
  int rc = sc_transcript_words(field, expr, num_rounds, &need);
  if (rc) return rc;
  if (!transcript) return fail(SC_ERR_INVALID, "NULL transcript");
  if (challenge_mode < SC_CHALLENGE_SHA3 || challenge_mode > SC_CHALLENGE_EXPLICIT)
    return fail(SC_ERR_INVALID, "unknown challenge mode %d", challenge_mode);
  if (words < need) return fail(SC_ERR_INVALID, "transcript needs %llu words, got %llu",
                                static_cast<unsigned long long>(need), static_cast<unsigned long long>(words));
  std::memset(transcript, 0, need * 4);
  transcript_header(transcript, field->hf, *expr, num_rounds, challenge_mode, 0, tables_tag);
  return SC_OK;
}

int sc_transcript_info(const uint32_t* transcript, uint64_t words, int* out_num_rounds, int* out_rounds_done,
                       int* out_challenge_mode, uint64_t* out_tables_tag) {
  TranscriptInfo I;
  int rc = transcript_parse(transcript, words, &I);
  if (rc) return rc;
  if (out_num_rounds) *out_num_rounds = I.n;
  if (out_rounds_done) *out_rounds_done = I.done;
  if (out_challenge_mode) *out_challenge_mode = I.mode;
  if (out_tables_tag) *out_tables_tag = I.tag;
  return SC_OK;
}

int sc_transcript_result(const sc_field* field, const sc_expr* expr, const uint32_t* transcript, uint64_t words,
                         uint32_t* out_round_polys, uint32_t* out_challenges, uint32_t* out_finals,
                         uint32_t* out_claim0, uint64_t* out_checksum) {
  if (!field || !expr) return fail(SC_ERR_INVALID, "NULL argument");
  TranscriptInfo I;
  int rc = transcript_parse(transcript, words, &I);
  if (!rc) rc = transcript_match(I, field->hf, *expr);
  if (rc) return rc;
  if (I.done < I.n) return fail(SC_ERR_PENDING, "transcript has %d of %d rounds", I.done, I.n);
  const int L = I.L, d = I.d, n = I.n;
  const StateOffsets so = state_offsets(n, I.K, L);
  const uint32_t* hs = transcript + kTranscriptHeader;
  if (out_round_polys)
    for (int j = 0; j < n; ++j)
      std::memcpy(out_round_polys + static_cast<size_t>(j) * (d + 1) * L, hs + so.polys + static_cast<size_t>(j) * kMaxPoints * L,
                  static_cast<size_t>(d + 1) * L * 4);
  if (out_challenges) std::memcpy(out_challenges, hs + so.chals, static_cast<size_t>(n) * L * 4);
  if (out_finals) std::memcpy(out_finals, hs + so.finals, static_cast<size_t>(1 + I.K) * L * 4);
  if (out_claim0) std::memcpy(out_claim0, hs + so.claim0, static_cast<size_t>(L) * 4);
  if (out_checksum) std::memcpy(out_checksum, hs + so.checksum, 8);
  return SC_OK;
}

int sc_tables_tag(int num_tables, const int32_t* table_kinds, uint64_t seed, uint64_t* out_tag) {
  if (!table_kinds || !out_tag) return fail(SC_ERR_INVALID, "NULL argument");
  if (num_tables < 1 || num_tables > kMaxVars) return fail(SC_ERR_INVALID, "num_tables %d outside 1..%d", num_tables, kMaxVars);
  *out_tag = seeded_tables_tag(num_tables, table_kinds, seed);
  return SC_OK;
}

int sc_prove_resume(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, const uint32_t* tables_dev,
                    const uint32_t* explicit_challenges, int stop_round, uint32_t* transcript, uint64_t words) {
  if (!ctx || !field || !expr || !tables_dev) return fail(SC_ERR_INVALID, "NULL argument");
  TranscriptInfo I;
  int rc = transcript_parse(transcript, words, &I);
  if (!rc) rc = transcript_match(I, field->hf, *expr);
  if (rc) return rc;
  if (I.done == I.n) return fail(SC_ERR_INVALID, "the transcript's proof is complete");
  if (stop_round <= I.done || stop_round > I.n)
    return fail(SC_ERR_INVALID, "stop_round %d outside %d..%d", stop_round, I.done + 1, I.n);
  if (reinterpret_cast<uintptr_t>(tables_dev) % 16) return fail(SC_ERR_INVALID, "tables_dev must be 16-byte aligned");
  if (field->device != ctx->device)
    return fail(SC_ERR_INVALID, "field was set up on device %d, context is on %d", field->device, ctx->device);
  uint32_t* state = transcript + kTranscriptHeader;
  const StateOffsets so = state_offsets(I.n, I.K, I.L);
  if (state[so.counter] || state[so.status]) return fail(SC_ERR_INVALID, "transcript state records a device error");
  if (I.mode == SC_CHALLENGE_EXPLICIT) {
    if (!explicit_challenges) return fail(SC_ERR_INVALID, "explicit challenge mode needs explicit_challenges");
    if (std::memcmp(explicit_challenges, state + so.chals, static_cast<size_t>(I.done) * I.L * 4))
      return fail(SC_ERR_INVALID, "explicit challenges differ from the transcript's first %d", I.done);
  }
  rc = prove_segment(ctx, field, expr, I.n, tables_dev, I.mode, explicit_challenges, I.done, stop_round, state);
  if (rc) return rc;
  transcript[kTwDone] = static_cast<uint32_t>(stop_round);
  return SC_OK;
}

}  // extern "C"
