// Batched proving: many independent proofs of one field in one CUDA graph.
//
// Proof p (num_rounds n_p) does its round t in tick t. The proofs of a batch are split by
// degree class (the kernel's register arrays are sized by the class), and every class runs
// its own sequence of ticks on its own stream. A tick is one launch of
// batch_round_kernel<L, K, DMAX> over a work queue of (proof round, tile) items built here on
// the host: a round of P pairs is cut into ceil(P / tile) items, tile = threads x pairs per
// thread. The whole batch -- state reset, the classes' ticks (forked onto their streams and
// joined), the copy of all proof states to pinned host memory -- is captured once into a
// CUDA graph and replayed by every sc_batch_run. The reference has no batching (every proof
// runs alone, with a blocking copy per interpolation point: cuda/src/field_sumcheck.cu:1012-1088).
#include <algorithm>
#include <vector>

#include "host_common.h"

using namespace sc;
using namespace sc_host;

namespace {
// Rounds with at least this many pairs derive g(1) from the claim (see capi.cu).
constexpr uint64_t kBatchSkip1MinPairs = uint64_t{1} << 12;
// Tail rounds (batch_round_kernel: from a proof's first one-tile round on, that item's block
// proves the rest of the proof) are off in batches. Measured on B200 with the 512-proof mixed
// stream: 9.0k proofs/s with tails, 9.9k without. A 256-bit tail of ~10 rounds takes a block
// ~200 us, longer than the late ticks it replaces (~30-45 us each), and every late tick then
// holds some proof's tail; without tails the proofs' small rounds overlap within each tick.
#ifndef SC_BATCH_TAILS
#define SC_BATCH_TAILS 0
#endif
constexpr bool kBatchTails = SC_BATCH_TAILS != 0;
#ifndef SC_BATCH_DMAX6
#define SC_BATCH_DMAX6 1
#endif
constexpr bool kBatchDmax6 = SC_BATCH_DMAX6 != 0;  // see dispatch_dmax

// Tails for fields of at most this many limbs only (0: none).
#ifndef SC_BATCH_TAIL_MAX_L
#define SC_BATCH_TAIL_MAX_L 0
#endif

// Ticks proof p takes: one per round, or up to its first one-tile round with tails.
inline int proof_ticks(int n, uint64_t tile, int L) {
  if (kBatchTails || L <= SC_BATCH_TAIL_MAX_L) {
    for (int t = 0; t < n; ++t)
      if ((uint64_t{1} << n) >> (t + 1) <= tile) return t + 1;
  }
  return n;
}

struct BatchClass {
  int dclass = 2;
  int dmax = 2;  // the kernel instance: dclass, or 6 for a degree <= 7 class without degree 7
  std::vector<int> proofs;
  int threads = 256;
  int grid = 1;
  size_t smem = 0;
  int max_rounds = 0;
  std::vector<int> tick_round0, tick_item0, tick_items;  // offsets into the batch's arrays
  int head0 = 0;                                         // this class's first queue counter
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<cudaEvent_t> tick_events;                  // around every tick, inside the graph
};
}  // namespace

struct sc_batch {
  sc_ctx* ctx = nullptr;
  const sc_field* field = nullptr;
  int L = 0, kind = 0;
  int count = 0;
  int mode = 0;
  int class_threads[3] = {0, 0, 0};  // requested threads per block, degree classes 2, 4, 7 (0: default)
  std::vector<int> ppt;               // pairs per thread of each proof's tiles
  std::vector<int> n, K, d;
  std::vector<StateOffsets> so;
  std::vector<size_t> state_base;  // word offset of each proof's state
  size_t state_words = 0;
  std::vector<BatchClass> classes;
  int total_heads = 0;
  DevBuf fold_pool, state, partials, rounds, items, heads, exprs;
  uint32_t* host_state = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ready = nullptr, done = nullptr, fork = nullptr;
  cudaEvent_t origin = nullptr;  // timing origin of a run (recorded inside the graph)
  cudaGraphExec_t exec = nullptr;
};

namespace {

template <int L, int K, int D>
struct KernelSetup {
  static int run(int kmax, int threads_req, int sm_count, int* threads_out, int* grid_out, size_t* smem_out) {

    int threads = std::min(threads_req ? threads_req : kernel_threads(L), kernel_threads(L));
    const int per_thread = round_smem_words_per_thread(kmax, L) * 4;
    while (threads > 32 && static_cast<size_t>(threads) * per_thread > static_cast<size_t>(kMaxDynSmem)) threads -= 32;
    const size_t smem = static_cast<size_t>(threads) * per_thread;
    SC_CUDA(cudaFuncSetAttribute(batch_round_kernel<L, K, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem));
    int bps = 0;
    SC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, batch_round_kernel<L, K, D>, threads, smem));
    if (bps < 1) return fail(SC_ERR_UNSUPPORTED, "batch kernel does not fit on an SM (tables=%d, L=%d)", kmax, L);
    *threads_out = threads;
    *grid_out = bps * sm_count;
    *smem_out = smem;
    return SC_OK;
  }
};

template <int L, int K, int D>
struct KernelLaunch {
  static int run(const sc_field* field, unsigned grid, int threads, size_t smem, cudaStream_t stream,
                 const BatchTickArgs& T) {
    FieldParams<L, K> F;
    for (int l = 0; l < L; ++l) F.p[l] = field->hf.p[l];
    F.np = field->hf.np;
    batch_round_kernel<L, K, D><<<grid, threads, smem, stream>>>(T, F);
    SC_CUDA(cudaGetLastError());
    return SC_OK;
  }
};

// The batched kernel's register arrays by the largest degree it proves: 2, 4, 6 or 7. A batch's
// degree <= 7 class whose proofs all have degree <= 6 runs the 6 instance, one point fewer:
// fewer registers and spills at 8 limbs (1192 -> 832 bytes of spill stores); measured on
// B200, the 512-proof mixed stream (degree <= 6), tuned: 10.30-10.33k -> 10.40k proofs/s.
template <template <int, int, int> class Fn, int L, int K, typename... Args>
inline int dispatch_dmax_l(int dmax, Args&&... args) {
  switch (dmax) {
    case 2: return Fn<L, K, 2>::run(args...);
    case 4: return Fn<L, K, 4>::run(args...);
    case 6: return Fn<L, K, 6>::run(args...);
    default: return Fn<L, K, 7>::run(args...);
  }
}

template <template <int, int, int> class Fn, typename... Args>
inline int dispatch_dmax(int L, int K, int dmax, Args&&... args) {
  switch (L) {
    case 1: return dispatch_dmax_l<Fn, 1, kFieldGeneric>(dmax, args...);
    case 2:
      return K == kFieldGoldilocks ? dispatch_dmax_l<Fn, 2, kFieldGoldilocks>(dmax, args...)
                                   : dispatch_dmax_l<Fn, 2, kFieldGeneric>(dmax, args...);
    case 4:
      return K == kFieldMersenne127 ? dispatch_dmax_l<Fn, 4, kFieldMersenne127>(dmax, args...)
                                    : dispatch_dmax_l<Fn, 4, kFieldGeneric>(dmax, args...);
    default: return dispatch_dmax_l<Fn, 8, kFieldGeneric>(dmax, args...);
  }
}

}  // namespace

namespace sc_host {

int batch_kernel_setup(int L, int K, int dmax, int kmax, int threads_req, int sm_count, int* threads, int* grid,
                       size_t* smem) {
  return dispatch_dmax<KernelSetup>(L, K, dmax, kmax, threads_req, sm_count, threads, grid, smem);
}

int batch_kernel_launch(int L, int K, int dmax, const sc_field* field, unsigned grid, int threads, size_t smem,
                        cudaStream_t stream, const BatchTickArgs& T) {
  return dispatch_dmax<KernelLaunch>(L, K, dmax, field, grid, threads, smem, stream, T);
}

}  // namespace sc_host

namespace {

int batch_tick(sc_batch* B, const BatchClass& C, int t, const BatchTickArgs& T) {
  const unsigned grid = static_cast<unsigned>(std::min(C.grid, std::max(1, T.num_items)));
  SC_CUDA(cudaEventRecordWithFlags(C.tick_events[2 * t], C.stream, cudaEventRecordExternal));
  const int rc = batch_kernel_launch(B->L, B->kind, C.dmax, B->field, grid, C.threads, C.smem, C.stream, T);
  if (rc) return rc;
  SC_CUDA(cudaEventRecordWithFlags(C.tick_events[2 * t + 1], C.stream, cudaEventRecordExternal));
  return SC_OK;
}

template <int L>
int batch_setup(sc_batch* B, const sc_expr* const* exprs, const uint32_t* const* tables) {
  sc_ctx* ctx = B->ctx;
  const int count = B->count;
  int rc;
  std::vector<ExprDev> ed(count);
  for (int p = 0; p < count; ++p) {
    build_expr_dev<L>(*exprs[p], *B->field, ed[p]);
    B->K.push_back(exprs[p]->num_vars);
    B->d.push_back(exprs[p]->degree);
  }
  // degree classes
  for (int dc : {2, 4, 7}) {
    BatchClass C;
    C.dclass = dc;
    int kmax = 1;
    for (int p = 0; p < count; ++p)
      if (degree_class(B->d[p]) == dc) {
        C.proofs.push_back(p);
        kmax = std::max(kmax, B->K[p]);
        C.max_rounds = std::max(C.max_rounds, B->n[p]);
      }
    if (C.proofs.empty()) continue;
    const int ci = dc == 2 ? 0 : (dc == 4 ? 1 : 2);
    int dmax_seen = 0;
    for (int p : C.proofs) dmax_seen = std::max(dmax_seen, B->d[p]);
    C.dmax = (kBatchDmax6 && dc == 7 && dmax_seen <= 6) ? 6 : dc;
    if ((rc = batch_kernel_setup(L, B->kind, C.dmax, kmax, B->class_threads[ci], ctx->sm_count, &C.threads, &C.grid,
                                 &C.smem)))
      return rc;
    C.max_rounds = 0;  // ticks of the class
    for (int p : C.proofs)
      C.max_rounds = std::max(C.max_rounds, proof_ticks(B->n[p], static_cast<uint64_t>(C.threads) * B->ppt[p], B->L));
    B->classes.push_back(std::move(C));
  }
  // per-proof state and fold buffers (16-byte aligned carve-outs of two pools)
  std::vector<size_t> fold_a(count), fold_b(count);
  size_t fold_words = 0;
  for (int p = 0; p < count; ++p) {
    const uint64_t N = uint64_t{1} << B->n[p];
    B->so.push_back(state_offsets(B->n[p], B->K[p], L));
    B->state_base.push_back(B->state_words);
    B->state_words += (B->so[p].total_words + 3) & ~size_t{3};
    fold_a[p] = fold_words;
    fold_words += (B->n[p] >= 2 ? static_cast<size_t>(B->K[p]) * L * (N / 2) : 0) + 4;
    fold_b[p] = fold_words;
    fold_words += (B->n[p] >= 3 ? static_cast<size_t>(B->K[p]) * L * (N / 4) : 0) + 4;
    fold_words = (fold_words + 3) & ~size_t{3};
  }
  if ((rc = ensure(ctx, B->fold_pool, fold_words * 4))) return rc;
  if ((rc = ensure(ctx, B->state, B->state_words * 4))) return rc;
  SC_CUDA(cudaMallocHost(&B->host_state, B->state_words * 4));
  uint32_t* st = static_cast<uint32_t*>(B->state.p);
  uint32_t* pool = static_cast<uint32_t*>(B->fold_pool.p);
  if ((rc = ensure(ctx, B->exprs, ed.size() * sizeof(ExprDev)))) return rc;
  const ExprDev* exprs_dev = static_cast<const ExprDev*>(B->exprs.p);
  // every class's ticks: rounds and items, in one array each (class and tick offsets)
  std::vector<BatchRound> rounds;
  std::vector<size_t> partial_item;  // per round: index of its first partial slot
  std::vector<BatchItem> items;
  for (BatchClass& C : B->classes) {
    C.head0 = B->total_heads;
    B->total_heads += C.max_rounds;
    for (int t = 0; t < C.max_rounds; ++t) {
      C.tick_round0.push_back(static_cast<int>(rounds.size()));
      C.tick_item0.push_back(static_cast<int>(items.size()));
      int tick_items = 0;
      for (int p : C.proofs) {
        const uint64_t tile = static_cast<uint64_t>(C.threads) * B->ppt[p];
        const int ticks = proof_ticks(B->n[p], tile, B->L);
        if (t >= ticks) continue;
        const int n = B->n[p];
        const uint64_t N = uint64_t{1} << n;
        BatchRound R;
        std::memset(&R, 0, sizeof(R));
        RoundArgs& A = R.args;
        A.round = t;
        A.num_rounds = n;
        A.mode = B->mode;
        A.fc = B->field->dev;
        A.pairs = N >> (t + 1);
        A.skip1 = (t >= 1 && A.pairs >= kBatchSkip1MinPairs) ? 1 : 0;
        A.want_claim = (t + 1 < n && (N >> (t + 2)) >= kBatchSkip1MinPairs) ? 1 : 0;
        if (t == 0) {
          A.fold = 0;
          A.src = tables[p];
          A.src_len = N;
        } else {
          A.fold = 1;
          A.src_len = N >> (t - 1);
          A.src = t == 1 ? tables[p] : pool + ((t & 1) ? fold_b[p] : fold_a[p]);
          A.dst = pool + ((t & 1) ? fold_a[p] : fold_b[p]);
        }
        uint32_t* s = st + B->state_base[p];
        const StateOffsets& o = B->so[p];
        A.st.counter = s + o.counter;
        A.st.status = s + o.status;
        A.st.checksum = reinterpret_cast<uint64_t*>(s + o.checksum);
        A.st.polys = s + o.polys;
        A.st.chals = s + o.chals;
        A.st.finals = s + o.finals;
        A.st.claim0 = s + o.claim0;
        A.st.claim = s + o.claim;
        R.expr = exprs_dev + p;
        if (t == ticks - 1 && ticks < n) {
          R.tail_rounds = n - ticks;
          R.skip1_min_pairs = static_cast<uint32_t>(kBatchSkip1MinPairs);
          R.fold_a = pool + fold_a[p];
          R.fold_b = pool + fold_b[p];
        }
        const uint64_t nitems = (A.pairs + tile - 1) / tile;
        R.first_item = static_cast<int>(items.size()) - C.tick_item0[t];  // tick-relative
        R.num_items = static_cast<int>(nitems);
        R.item_base = 0;
        R.round_items = static_cast<int>(nitems);
        partial_item.push_back(items.size());
        const int ridx = static_cast<int>(rounds.size()) - C.tick_round0[t];
        for (uint64_t i = 0; i < nitems; ++i) {
          BatchItem I;
          I.round = ridx;
          I.pad = 0;
          I.start = i * tile;
          I.count = std::min<uint64_t>(tile, A.pairs - i * tile);
          items.push_back(I);
        }
        rounds.push_back(R);
        tick_items += static_cast<int>(nitems);
      }
      C.tick_items.push_back(tick_items);
    }
  }
  if ((rc = ensure(ctx, B->partials, items.size() * kMaxPoints * L * 4))) return rc;
  if ((rc = ensure(ctx, B->rounds, rounds.size() * sizeof(BatchRound)))) return rc;
  if ((rc = ensure(ctx, B->items, items.size() * sizeof(BatchItem)))) return rc;
  if ((rc = ensure(ctx, B->heads, static_cast<size_t>(std::max(1, B->total_heads)) * 4))) return rc;
  for (size_t r = 0; r < rounds.size(); ++r)
    rounds[r].partials = static_cast<uint32_t*>(B->partials.p) + partial_item[r] * kMaxPoints * L;
  SC_CUDA(cudaMemcpy(B->rounds.p, rounds.data(), rounds.size() * sizeof(BatchRound), cudaMemcpyHostToDevice));
  SC_CUDA(cudaMemcpy(B->items.p, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice));
  SC_CUDA(cudaMemcpy(B->exprs.p, ed.data(), ed.size() * sizeof(ExprDev), cudaMemcpyHostToDevice));
  return SC_OK;
}

// The launch sequence of one run (captured once into the graph).
int batch_issue(sc_batch* B) {
  SC_CUDA(cudaMemsetAsync(B->state.p, 0, B->state_words * 4, B->stream));
  SC_CUDA(cudaMemsetAsync(B->heads.p, 0, static_cast<size_t>(std::max(1, B->total_heads)) * 4, B->stream));
  SC_CUDA(cudaEventRecordWithFlags(B->origin, B->stream, cudaEventRecordExternal));
  SC_CUDA(cudaEventRecord(B->fork, B->stream));
  for (BatchClass& C : B->classes) {
    SC_CUDA(cudaStreamWaitEvent(C.stream, B->fork, 0));
    for (int t = 0; t < C.max_rounds; ++t) {
      BatchTickArgs T;
      T.rounds = static_cast<const BatchRound*>(B->rounds.p) + C.tick_round0[t];
      T.items = static_cast<const BatchItem*>(B->items.p) + C.tick_item0[t];
      T.num_items = C.tick_items[t];
      T.pad = 0;
      T.head = static_cast<uint32_t*>(B->heads.p) + C.head0 + t;
      T.tile = 0;
      const int rc = batch_tick(B, C, t, T);
      if (rc) return rc;
    }
    SC_CUDA(cudaEventRecord(C.done, C.stream));
    SC_CUDA(cudaStreamWaitEvent(B->stream, C.done, 0));
  }
  SC_CUDA(cudaMemcpyAsync(B->host_state, B->state.p, B->state_words * 4, cudaMemcpyDeviceToHost, B->stream));
  return SC_OK;
}

}  // namespace

extern "C" {

int sc_batch_create_tiled(sc_ctx* ctx, const sc_field* field, int count, const sc_expr* const* exprs,
                          const int32_t* num_rounds, const uint32_t* const* tables_dev, int challenge_mode,
                          const int32_t* class_threads, const int32_t* proof_pairs_per_thread, sc_batch** out) {
  if (!ctx || !field || !exprs || !num_rounds || !tables_dev || !out) return fail(SC_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (count < 1) return fail(SC_ERR_INVALID, "empty batch");
  if (challenge_mode != SC_CHALLENGE_SHA3 && challenge_mode != SC_CHALLENGE_FIXED)
    return fail(SC_ERR_INVALID, "batches derive their challenges: SHA3 or fixed mode");
  for (int c = 0; class_threads && c < 3; ++c)
    if (class_threads[c] != 0 && (class_threads[c] < 32 || class_threads[c] > 256 || class_threads[c] % 32))
      return fail(SC_ERR_INVALID, "class_threads[%d] must be 0 (auto) or a multiple of 32 in 32..256", c);
  for (int p = 0; proof_pairs_per_thread && p < count; ++p)
    if (proof_pairs_per_thread[p] < 0 || proof_pairs_per_thread[p] > 64)
      return fail(SC_ERR_INVALID, "proof %d: pairs_per_thread outside 0..64", p);
  for (int p = 0; p < count; ++p) {
    if (!exprs[p] || !tables_dev[p]) return fail(SC_ERR_INVALID, "proof %d: NULL expression or tables", p);
    if (num_rounds[p] < 1 || num_rounds[p] > kMaxRounds) return fail(SC_ERR_INVALID, "proof %d: num_rounds %d", p, num_rounds[p]);
    if (reinterpret_cast<uintptr_t>(tables_dev[p]) % 16) return fail(SC_ERR_INVALID, "proof %d: tables not 16-byte aligned", p);
  }
  SC_CUDA(cudaSetDevice(ctx->device));
  sc_batch* B = new (std::nothrow) sc_batch();
  if (!B) return fail(SC_ERR_NOMEM, "host allocation failed");
  B->ctx = ctx;
  B->field = field;
  B->L = field->hf.L;
  B->kind = field_kind(field->hf.p, B->L);
  B->count = count;
  B->mode = challenge_mode;
  for (int c = 0; c < 3; ++c) B->class_threads[c] = class_threads ? class_threads[c] : 0;
  for (int p = 0; p < count; ++p) {
    const int v = proof_pairs_per_thread ? proof_pairs_per_thread[p] : 0;
    B->ppt.push_back(v ? v : 2);
  }
  for (int p = 0; p < count; ++p) B->n.push_back(num_rounds[p]);
  int rc;
  switch (B->L) {
    case 1: rc = batch_setup<1>(B, exprs, tables_dev); break;
    case 2: rc = batch_setup<2>(B, exprs, tables_dev); break;
    case 4: rc = batch_setup<4>(B, exprs, tables_dev); break;
    default: rc = batch_setup<8>(B, exprs, tables_dev); break;
  }
  cudaError_t e = cudaSuccess;
  if (!rc) e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
  if (!rc && e == cudaSuccess) e = cudaEventCreateWithFlags(&B->ready, cudaEventDisableTiming);
  if (!rc && e == cudaSuccess) e = cudaEventCreateWithFlags(&B->done, cudaEventDisableTiming);
  if (!rc && e == cudaSuccess) e = cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming);
  if (!rc && e == cudaSuccess) e = cudaEventCreate(&B->origin);
  for (size_t c = 0; !rc && e == cudaSuccess && c < B->classes.size(); ++c) {
    BatchClass& C = B->classes[c];
    e = cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&C.done, cudaEventDisableTiming);
    for (int i = 0; e == cudaSuccess && i < 2 * C.max_rounds; ++i) {
      cudaEvent_t ev;
      e = cudaEventCreate(&ev);
      if (e == cudaSuccess) C.tick_events.push_back(ev);
    }
  }
  if (!rc && e != cudaSuccess) rc = fail(SC_ERR_CUDA, "batch streams/events: %s", cudaGetErrorString(e));
  if (rc) {
    sc_batch_destroy(B);
    return rc;
  }
  *out = B;
  return SC_OK;
}

int sc_batch_create(sc_ctx* ctx, const sc_field* field, int count, const sc_expr* const* exprs,
                    const int32_t* num_rounds, const uint32_t* const* tables_dev, int challenge_mode,
                    int threads, int pairs_per_thread, sc_batch** out) {
  if (threads != 0 && (threads < 32 || threads > 256 || threads % 32))
    return fail(SC_ERR_INVALID, "threads must be 0 (auto) or a multiple of 32 in 32..256");
  if (pairs_per_thread < 0 || pairs_per_thread > 64) return fail(SC_ERR_INVALID, "pairs_per_thread outside 0..64");
  if (count < 1) return fail(SC_ERR_INVALID, "empty batch");
  const int32_t ct[3] = {threads, threads, threads};
  std::vector<int32_t> ppt(static_cast<size_t>(count), pairs_per_thread);
  return sc_batch_create_tiled(ctx, field, count, exprs, num_rounds, tables_dev, challenge_mode, ct, ppt.data(), out);
}

int sc_batch_launch(sc_batch* B) {
  if (!B) return fail(SC_ERR_INVALID, "NULL batch");
  SC_CUDA(cudaSetDevice(B->ctx->device));
  // the batch starts after the work already queued on the caller's stream
  SC_CUDA(cudaEventRecord(B->ready, B->ctx->stream));
  SC_CUDA(cudaStreamWaitEvent(B->stream, B->ready, 0));
  if (!B->exec) {
    cudaGraph_t g = nullptr;
    SC_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_issue(B);
    cudaError_t e = cudaStreamEndCapture(B->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return fail(SC_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&B->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(SC_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  }
  SC_CUDA(cudaGraphLaunch(B->exec, B->stream));
  SC_CUDA(cudaEventRecord(B->done, B->stream));
  return SC_OK;
}

int sc_batch_join(sc_batch* B) {
  if (!B) return fail(SC_ERR_INVALID, "NULL batch");
  SC_CUDA(cudaSetDevice(B->ctx->device));
  SC_CUDA(cudaStreamWaitEvent(B->ctx->stream, B->done, 0));
  return SC_OK;
}

int sc_batch_run(sc_batch* B) {
  const int rc = sc_batch_launch(B);
  return rc ? rc : sc_batch_join(B);
}

int sc_batch_wait(sc_batch* B) {
  if (!B) return fail(SC_ERR_INVALID, "NULL batch");
  SC_CUDA(cudaEventSynchronize(B->done));
  for (int p = 0; p < B->count; ++p)
    if (B->host_state[B->state_base[p] + B->so[p].status])
      return fail(SC_ERR_DEVICE, "proof %d: device status %u", p, B->host_state[B->state_base[p] + B->so[p].status]);
  return SC_OK;
}

int sc_batch_tick_times(sc_batch* B, float* out_start_ms, float* out_end_ms, int capacity, int* count) {
  if (!B || !count) return fail(SC_ERR_INVALID, "NULL argument");
  int k = 0;
  for (const BatchClass& C : B->classes) k += C.max_rounds;
  *count = k;
  int i = 0;
  for (const BatchClass& C : B->classes)
    for (int t = 0; t < C.max_rounds; ++t, ++i) {
      if (i >= capacity) continue;
      float a = 0.f, b = 0.f;
      SC_CUDA(cudaEventElapsedTime(&a, B->origin, C.tick_events[2 * t]));
      SC_CUDA(cudaEventElapsedTime(&b, B->origin, C.tick_events[2 * t + 1]));
      if (out_start_ms) out_start_ms[i] = a;
      if (out_end_ms) out_end_ms[i] = b;
    }
  return SC_OK;
}

int sc_batch_classes(sc_batch* B, int32_t* out_degree_class, int32_t* out_ticks, int capacity, int* count) {
  if (!B || !count) return fail(SC_ERR_INVALID, "NULL argument");
  *count = static_cast<int>(B->classes.size());
  for (int c = 0; c < *count && c < capacity; ++c) {
    if (out_degree_class) out_degree_class[c] = B->classes[c].dclass;
    if (out_ticks) out_ticks[c] = B->classes[c].max_rounds;
  }
  return SC_OK;
}

int sc_batch_class_proofs(sc_batch* B, int cls, int32_t* out_indices, int capacity, int* count) {
  if (!B || !count) return fail(SC_ERR_INVALID, "NULL argument");
  if (cls < 0 || cls >= static_cast<int>(B->classes.size())) return fail(SC_ERR_INVALID, "class %d", cls);
  const auto& v = B->classes[cls].proofs;
  *count = static_cast<int>(v.size());
  for (int i = 0; out_indices && i < *count && i < capacity; ++i) out_indices[i] = v[i];
  return SC_OK;
}

int sc_batch_result(sc_batch* B, int index, uint32_t* out_round_polys, uint32_t* out_challenges,
                    uint32_t* out_finals, uint32_t* out_claim0, uint64_t* out_checksum) {
  if (!B) return fail(SC_ERR_INVALID, "NULL batch");
  if (index < 0 || index >= B->count) return fail(SC_ERR_INVALID, "index %d outside 0..%d", index, B->count - 1);
  const int L = B->L, n = B->n[index], d = B->d[index], K = B->K[index];
  const uint32_t* hs = B->host_state + B->state_base[index];
  const StateOffsets& so = B->so[index];
  if (out_round_polys)
    for (int j = 0; j < n; ++j)
      std::memcpy(out_round_polys + static_cast<size_t>(j) * (d + 1) * L, hs + so.polys + static_cast<size_t>(j) * kMaxPoints * L,
                  static_cast<size_t>(d + 1) * L * 4);
  if (out_challenges) std::memcpy(out_challenges, hs + so.chals, static_cast<size_t>(n) * L * 4);
  if (out_finals) std::memcpy(out_finals, hs + so.finals, static_cast<size_t>(1 + K) * L * 4);
  if (out_claim0) std::memcpy(out_claim0, hs + so.claim0, L * 4);
  if (out_checksum) std::memcpy(out_checksum, hs + so.checksum, 8);
  return SC_OK;
}

int sc_batch_results(sc_batch* B, uint32_t* out_round_polys, uint32_t* out_challenges, uint32_t* out_finals,
                     uint32_t* out_claim0, uint64_t* out_checksums) {
  if (!B) return fail(SC_ERR_INVALID, "NULL batch");
  const int L = B->L;
  size_t op = 0, oc = 0, of = 0;
  for (int p = 0; p < B->count; ++p) {
    const int n = B->n[p], d = B->d[p], K = B->K[p];
    int rc = sc_batch_result(B, p, out_round_polys ? out_round_polys + op : nullptr,
                             out_challenges ? out_challenges + oc : nullptr, out_finals ? out_finals + of : nullptr,
                             out_claim0 ? out_claim0 + static_cast<size_t>(p) * L : nullptr,
                             out_checksums ? out_checksums + p : nullptr);
    if (rc) return rc;
    op += static_cast<size_t>(n) * (d + 1) * L;
    oc += static_cast<size_t>(n) * L;
    of += static_cast<size_t>(1 + K) * L;
  }
  return SC_OK;
}

int sc_batch_destroy(sc_batch* B) {
  if (!B) return SC_OK;
  cudaSetDevice(B->ctx->device);
  if (B->stream) cudaStreamSynchronize(B->stream);
  if (B->exec) cudaGraphExecDestroy(B->exec);
  for (DevBuf* b : {&B->fold_pool, &B->state, &B->partials, &B->rounds, &B->items, &B->heads, &B->exprs})
    if (b->p) cudaFree(b->p);
  if (B->host_state) cudaFreeHost(B->host_state);
  for (BatchClass& C : B->classes) {
    for (cudaEvent_t e : C.tick_events) cudaEventDestroy(e);
    if (C.done) cudaEventDestroy(C.done);
    if (C.stream) cudaStreamDestroy(C.stream);
  }
  if (B->ready) cudaEventDestroy(B->ready);
  if (B->done) cudaEventDestroy(B->done);
  if (B->fork) cudaEventDestroy(B->fork);
  if (B->origin) cudaEventDestroy(B->origin);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
  return SC_OK;
}

}  // extern "C"
