// Batched proving: many independent proofs of one field in one CUDA graph.
//
// Proof p (num_rounds n_p) does its round t in tick t. A tick is one launch of
// batch_round_kernel<L> over a work queue of (proof round, tile) items built here on the
// host: a round of P pairs is cut into ceil(P / tile) items, tile = threads x pairs per
// thread. The whole batch -- state reset, every tick, the copy of all proof states to
// pinned host memory -- is captured once into a CUDA graph on the batch's own stream and
// replayed by every sc_batch_run. The reference has no batching (every proof runs alone,
// with a blocking copy per interpolation point: cuda/src/field_sumcheck.cu:1012-1088).
#include <algorithm>
#include <vector>

#include "host_common.h"

using namespace sc;
using namespace sc_host;

struct sc_batch {
  sc_ctx* ctx = nullptr;
  const sc_field* field = nullptr;
  int L = 0;
  int count = 0;
  int mode = 0;
  int threads = 256;
  int grid = 0;
  size_t smem = 0;
  int max_rounds = 0;
  std::vector<int> n, K, d;
  std::vector<StateOffsets> so;
  std::vector<size_t> state_base;  // word offset of each proof's state
  size_t state_words = 0;
  std::vector<int> tick_round0, tick_rounds, tick_item0, tick_items;
  DevBuf fold_pool, state, partials, rounds, items, heads, exprs;
  uint32_t* host_state = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ready = nullptr, done = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<float> tick_ms;  // per-tick device time of the last run
  std::vector<cudaEvent_t> tick_events;  // recorded around every tick (inside the graph)
};

namespace {

template <int L>
int batch_setup(sc_batch* B, const sc_expr* const* exprs, const uint32_t* const* tables, int ppt) {
  sc_ctx* ctx = B->ctx;
  const int count = B->count;
  int rc;
  // expressions
  std::vector<ExprDev> ed(count);
  int kmax = 1;
  for (int p = 0; p < count; ++p) {
    build_expr_dev<L>(*exprs[p], *B->field, ed[p]);
    B->K.push_back(exprs[p]->num_vars);
    B->d.push_back(exprs[p]->degree);
    kmax = std::max(kmax, exprs[p]->num_vars);
  }
  // launch shape
  int threads = B->threads;
  const int per_thread = round_smem_words_per_thread(kmax, L) * 4;
  while (threads > 32 && static_cast<size_t>(threads) * per_thread > static_cast<size_t>(kMaxDynSmem)) threads -= 32;
  B->threads = threads;
  B->smem = static_cast<size_t>(threads) * per_thread;
  SC_CUDA(cudaFuncSetAttribute(batch_round_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem));
  int bps = 0;
  SC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, batch_round_kernel<L>, threads, B->smem));
  if (bps < 1) return fail(SC_ERR_UNSUPPORTED, "batch kernel does not fit on an SM (K=%d, L=%d)", kmax, L);
  B->grid = bps * ctx->sm_count;
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
  // ticks: rounds and items
  std::vector<BatchRound> rounds;
  std::vector<BatchItem> items;
  for (int t = 0; t < B->max_rounds; ++t) {
    B->tick_round0.push_back(static_cast<int>(rounds.size()));
    B->tick_item0.push_back(static_cast<int>(items.size()));
    int tick_rounds = 0, tick_items = 0;
    for (int p = 0; p < count; ++p) {
      if (t >= B->n[p]) continue;
      const uint64_t N = uint64_t{1} << B->n[p];
      BatchRound R;
      std::memset(&R, 0, sizeof(R));
      RoundArgs& A = R.args;
      A.round = t;
      A.num_rounds = B->n[p];
      A.mode = B->mode;
      A.fc = B->field->dev;
      A.pairs = N >> (t + 1);
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
      R.expr = p;
      const uint64_t tile = static_cast<uint64_t>(threads) * ppt;
      const uint64_t nitems = (A.pairs + tile - 1) / tile;
      R.first_item = static_cast<int>(items.size()) - B->tick_item0[t];  // tick-relative
      R.num_items = static_cast<int>(nitems);
      const int ridx = static_cast<int>(rounds.size()) - B->tick_round0[t];
      for (uint64_t i = 0; i < nitems; ++i) {
        BatchItem I;
        I.round = ridx;
        I.pad = 0;
        I.start = i * tile;
        I.count = std::min<uint64_t>(tile, A.pairs - i * tile);
        items.push_back(I);
      }
      rounds.push_back(R);
      ++tick_rounds;
      tick_items += static_cast<int>(nitems);
    }
    B->tick_rounds.push_back(tick_rounds);
    B->tick_items.push_back(tick_items);
  }
  // partial index = global item index
  if ((rc = ensure(ctx, B->partials, items.size() * kMaxPoints * L * 4))) return rc;
  if ((rc = ensure(ctx, B->rounds, rounds.size() * sizeof(BatchRound)))) return rc;
  if ((rc = ensure(ctx, B->items, items.size() * sizeof(BatchItem)))) return rc;
  if ((rc = ensure(ctx, B->heads, static_cast<size_t>(B->max_rounds) * 4))) return rc;
  if ((rc = ensure(ctx, B->exprs, ed.size() * sizeof(ExprDev)))) return rc;
  SC_CUDA(cudaMemcpy(B->rounds.p, rounds.data(), rounds.size() * sizeof(BatchRound), cudaMemcpyHostToDevice));
  SC_CUDA(cudaMemcpy(B->items.p, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice));
  SC_CUDA(cudaMemcpy(B->exprs.p, ed.data(), ed.size() * sizeof(ExprDev), cudaMemcpyHostToDevice));
  return SC_OK;
}

// The launch sequence of one run (captured once into the graph).
template <int L>
int batch_issue(sc_batch* B) {
  FieldParams<L> F;
  for (int l = 0; l < L; ++l) F.p[l] = B->field->hf.p[l];
  F.np = B->field->hf.np;
  SC_CUDA(cudaMemsetAsync(B->state.p, 0, B->state_words * 4, B->stream));
  SC_CUDA(cudaMemsetAsync(B->heads.p, 0, static_cast<size_t>(B->max_rounds) * 4, B->stream));
  for (int t = 0; t < B->max_rounds; ++t) {
    BatchTickArgs T;
    T.rounds = static_cast<const BatchRound*>(B->rounds.p) + B->tick_round0[t];
    T.items = static_cast<const BatchItem*>(B->items.p) + B->tick_item0[t];
    T.num_items = B->tick_items[t];
    T.pad = 0;
    T.head = static_cast<uint32_t*>(B->heads.p) + t;
    T.exprs = static_cast<const ExprDev*>(B->exprs.p);
    T.partials = static_cast<uint32_t*>(B->partials.p) + static_cast<size_t>(B->tick_item0[t]) * kMaxPoints * L;
    const unsigned grid = static_cast<unsigned>(std::min(B->grid, std::max(1, T.num_items)));
    SC_CUDA(cudaEventRecordWithFlags(B->tick_events[2 * t], B->stream, cudaEventRecordExternal));
    batch_round_kernel<L><<<grid, B->threads, B->smem, B->stream>>>(T, F);
    SC_CUDA(cudaGetLastError());
    SC_CUDA(cudaEventRecordWithFlags(B->tick_events[2 * t + 1], B->stream, cudaEventRecordExternal));
  }
  SC_CUDA(cudaMemcpyAsync(B->host_state, B->state.p, B->state_words * 4, cudaMemcpyDeviceToHost, B->stream));
  return SC_OK;
}

int batch_issue_any(sc_batch* B) {
  switch (B->L) {
    case 1: return batch_issue<1>(B);
    case 2: return batch_issue<2>(B);
    case 4: return batch_issue<4>(B);
    default: return batch_issue<8>(B);
  }
}

}  // namespace

extern "C" {

int sc_batch_create(sc_ctx* ctx, const sc_field* field, int count, const sc_expr* const* exprs,
                    const int32_t* num_rounds, const uint32_t* const* tables_dev, int challenge_mode,
                    int threads, int pairs_per_thread, sc_batch** out) {
  if (!ctx || !field || !exprs || !num_rounds || !tables_dev || !out) return fail(SC_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (count < 1) return fail(SC_ERR_INVALID, "empty batch");
  if (challenge_mode != SC_CHALLENGE_SHA3 && challenge_mode != SC_CHALLENGE_FIXED)
    return fail(SC_ERR_INVALID, "batches derive their challenges: SHA3 or fixed mode");
  if (threads != 0 && (threads < 32 || threads > 256 || threads % 32))
    return fail(SC_ERR_INVALID, "threads must be 0 (auto) or a multiple of 32 in 32..256");
  if (pairs_per_thread < 0 || pairs_per_thread > 64) return fail(SC_ERR_INVALID, "pairs_per_thread outside 0..64");
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
  B->count = count;
  B->mode = challenge_mode;
  B->threads = threads ? threads : 256;
  for (int p = 0; p < count; ++p) {
    B->n.push_back(num_rounds[p]);
    B->max_rounds = std::max(B->max_rounds, num_rounds[p]);
  }
  const int ppt = pairs_per_thread ? pairs_per_thread : 2;
  int rc;
  switch (B->L) {
    case 1: rc = batch_setup<1>(B, exprs, tables_dev, ppt); break;
    case 2: rc = batch_setup<2>(B, exprs, tables_dev, ppt); break;
    case 4: rc = batch_setup<4>(B, exprs, tables_dev, ppt); break;
    default: rc = batch_setup<8>(B, exprs, tables_dev, ppt); break;
  }
  cudaError_t e = cudaSuccess;
  if (!rc) e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
  for (int i = 0; !rc && e == cudaSuccess && i < 2 * B->max_rounds; ++i) {
    cudaEvent_t ev;
    e = cudaEventCreate(&ev);
    if (e == cudaSuccess) B->tick_events.push_back(ev);
  }
  if (!rc && e == cudaSuccess) e = cudaEventCreateWithFlags(&B->ready, cudaEventDisableTiming);
  if (!rc && e == cudaSuccess) e = cudaEventCreateWithFlags(&B->done, cudaEventDisableTiming);
  if (!rc && e != cudaSuccess) rc = fail(SC_ERR_CUDA, "batch stream/events: %s", cudaGetErrorString(e));
  if (rc) {
    sc_batch_destroy(B);
    return rc;
  }
  *out = B;
  return SC_OK;
}

int sc_batch_run(sc_batch* B) {
  if (!B) return fail(SC_ERR_INVALID, "NULL batch");
  SC_CUDA(cudaSetDevice(B->ctx->device));
  // the batch starts after the work already queued on the caller's stream
  SC_CUDA(cudaEventRecord(B->ready, B->ctx->stream));
  SC_CUDA(cudaStreamWaitEvent(B->stream, B->ready, 0));
  int rc;
  if (!B->exec) {
    cudaGraph_t g = nullptr;
    SC_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    rc = batch_issue_any(B);
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
  SC_CUDA(cudaStreamWaitEvent(B->ctx->stream, B->done, 0));
  return SC_OK;
}

int sc_batch_wait(sc_batch* B) {
  if (!B) return fail(SC_ERR_INVALID, "NULL batch");
  SC_CUDA(cudaEventSynchronize(B->done));
  B->tick_ms.assign(B->max_rounds, 0.f);
  for (int t = 0; t < B->max_rounds; ++t)
    SC_CUDA(cudaEventElapsedTime(&B->tick_ms[t], B->tick_events[2 * t], B->tick_events[2 * t + 1]));
  for (int p = 0; p < B->count; ++p)
    if (B->host_state[B->state_base[p] + B->so[p].status])
      return fail(SC_ERR_DEVICE, "proof %d: device status %u", p, B->host_state[B->state_base[p] + B->so[p].status]);
  return SC_OK;
}

int sc_batch_tick_times(sc_batch* B, float* out_ms, int capacity, int* count) {
  if (!B || !count) return fail(SC_ERR_INVALID, "NULL argument");
  *count = static_cast<int>(B->tick_ms.size());
  for (int i = 0; out_ms && i < *count && i < capacity; ++i) out_ms[i] = B->tick_ms[i];
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

int sc_batch_destroy(sc_batch* B) {
  if (!B) return SC_OK;
  cudaSetDevice(B->ctx->device);
  if (B->stream) cudaStreamSynchronize(B->stream);
  if (B->exec) cudaGraphExecDestroy(B->exec);
  for (DevBuf* b : {&B->fold_pool, &B->state, &B->partials, &B->rounds, &B->items, &B->heads, &B->exprs})
    if (b->p) cudaFree(b->p);
  if (B->host_state) cudaFreeHost(B->host_state);
  for (cudaEvent_t e : B->tick_events) cudaEventDestroy(e);
  if (B->ready) cudaEventDestroy(B->ready);
  if (B->done) cudaEventDestroy(B->done);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
  return SC_OK;
}

}  // extern "C"
