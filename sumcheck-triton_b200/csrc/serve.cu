// Served proving: a request loop with continuous batching under an HBM budget.
//
// One worker thread per server owns two streams, a device memory pool and the request state.
// Requests whose round 0 fills more than one wave of the GPU ("large") run whole on the
// large-proof lane, a low-priority stream: one launch per round, one block per tile, issued
// at admission. All others are batched continuously in ticks on high-priority streams, so
// their blocks are dispatched ahead of the lane's as the lane's blocks retire: small proofs
// overtake large ones on the device instead of queueing behind them, while a large proof
// runs at the efficiency of its own full-GPU rounds. Each iteration of the worker's loop
//   1. moves submitted requests into the arrival-order waiting queue;
//   2. admits requests from the head of that queue while the admitted footprint stays within
//      the budget: allocates the request's block from the pool (stream-ordered), uploads its
//      expression, generates its tables from the seed on the device -- all queued behind the
//      work already on the stream, so admission never waits for the GPU (a large request's
//      whole proof, result copy and free are queued on the lane right here);
//   3. issues one tick: (request round, tile) items of one batched-round-kernel launch per
//      degree class (classes on their own streams, forked from and joined back to the
//      server stream). Every request whose current round has at most one wave of tiles
//      left runs all of them; the larger rounds share the tick's budget (two waves by
//      default) oldest request first. A round larger than its share advances over several
//      ticks; its partial slots and ticket live in the request's block, so the launch
//      holding its last tile finalises it (SHA3 challenge included) wherever that falls. A
//      request whose last round was issued gets its state copied to pinned memory and its
//      block freed (both stream-ordered) in the same tick;
//   4. retires finished ticks and large requests (event queries) and publishes results.
// The host runs at most kSlots ticks ahead of the GPU; tick t+1 is built while tick t runs.
//
// The FIFO-plain policy is the baseline: one request at a time, tables generated, then the
// plain per-round path (sc_prove).
//
// Suspension: a request marked by sc_server_suspend leaves at its next round boundary -- the
// first tick that finds its current round not yet started issues nothing for it and instead
// queues its state copy and block free, as for a finished request -- and is published with
// SC_SUSPENDED and its state words (its transcript). A resumed request (submit_resume)
// starts from such a state: admission uploads it instead of zeroing, regenerates the tables
// from the seed and refolds them with the recorded challenges to the round it continues from.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "host_common.h"

using namespace sc;
using namespace sc_host;

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kSlots = 2;                       // ticks in flight at most
constexpr uint64_t kServeSkip1MinPairs = uint64_t{1} << 12;
// Once a request's round fits one tile, that item's block proves the rest of the proof
// (tail rounds, batch_round_kernel): one tick instead of one per remaining round. Measured
// on B200, 5,000 requests of the served stream at 80% load: p50 1.85 -> 1.42 ms, p90 14.3 ->
// 12.1 ms, p99 39.4 -> 36.0 ms, ticks 35.9k -> 14.2k. Tail items come first in their tick
// (phase 1 below), so they start while the larger rounds' items run.
#ifndef SC_SERVE_TAILS
#define SC_SERVE_TAILS 1
#endif
constexpr bool kServeTails = SC_SERVE_TAILS != 0;

void set_tail(BatchRound& B, const RoundArgs& A, uint32_t* fold_a, uint32_t* fold_b) {
  B.tail_rounds = A.num_rounds - 1 - A.round;
  B.skip1_min_pairs = static_cast<uint32_t>(kServeSkip1MinPairs);
  B.fold_a = fold_a;
  B.fold_b = fold_b;
}
constexpr size_t kAlign = 256;

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct ServeRequest {
  uint64_t id = 0;
  sc_expr expr;
  int n = 0, K = 0, d = 0, dclass = 2;
  std::vector<int32_t> kinds;
  uint64_t seed = 0;
  int mode = SC_CHALLENGE_SHA3;
  size_t footprint = 0;
  double t_submit = 0, t_admit = -1, t_done = -1;
  int status = SC_ERR_PENDING;  // guarded by the server mutex
  // results (written by the worker before status leaves PENDING)
  std::vector<uint32_t> polys, chals, finals, claim0;
  uint64_t checksum = 0;
  // transcripts: the round it starts from and that state (resumed requests); the suspend
  // mark; the state it was suspended with (state words, rounds done)
  int first = 0;
  std::vector<uint32_t> resume_state;
  std::atomic<bool> suspend{false};
  bool suspending = false;  // worker: leaving with this tick
  std::vector<uint32_t> suspended_state;
  int suspended_done = 0;
  // device residence (worker only)
  StateOffsets so{};
  char* block = nullptr;
  uint32_t* state = nullptr;
  uint32_t* partials = nullptr;
  ExprDev* expr_dev = nullptr;
  uint32_t* tables = nullptr;
  uint32_t* fold_a = nullptr;
  uint32_t* fold_b = nullptr;
  BatchRound* rounds_dev = nullptr;  // large requests: every round's descriptor
  bool large = false;    // runs whole on the large-proof lane
  int slot = -1;         // pinned staging slot
  int round = 0;         // current round
  uint64_t issued = 0;   // items of the current round issued so far
};

struct ServeClass {
  int dclass = 2;
  int threads = 256;
  int grid = 1;
  size_t smem = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
};

struct TickSlot {
  char* host = nullptr;  // pinned: heads, then per class rounds and items
  char* dev = nullptr;
  size_t cap = 0;
  cudaEvent_t done = nullptr;
  bool busy = false;
  std::vector<ServeRequest*> completing;
};

// Layout of one request's device block. Offsets in bytes, every part kAlign-aligned.
struct BlockLayout {
  size_t state, partials, expr, rounds, tables, fold_a, fold_b, total;
};

inline BlockLayout block_layout(int n, int K, int L, int tile_pairs) {
  const uint64_t N = uint64_t{1} << n;
  const uint64_t items0 = ((N >> 1) + tile_pairs - 1) / tile_pairs;
  BlockLayout b;
  size_t off = 0;
  b.state = off;
  off = align_up(off + state_offsets(n, K, L).total_words * 4, kAlign);
  b.partials = off;
  off = align_up(off + std::max<uint64_t>(items0, 1) * kMaxPoints * L * 4, kAlign);
  b.expr = off;
  off = align_up(off + sizeof(ExprDev), kAlign);
  b.rounds = off;
  off = align_up(off + static_cast<size_t>(n) * sizeof(BatchRound), kAlign);
  b.tables = off;
  off = align_up(off + static_cast<size_t>(K) * L * N * 4, kAlign);
  b.fold_a = off;
  off = align_up(off + (n >= 2 ? static_cast<size_t>(K) * L * (N / 2) * 4 : 0), kAlign);
  b.fold_b = off;
  off = align_up(off + (n >= 3 ? static_cast<size_t>(K) * L * (N / 4) * 4 : 0), kAlign);
  b.total = off;
  return b;
}

}  // namespace

struct sc_server {
  int device = 0;
  const sc_field* field = nullptr;
  int L = 0, kind = 0, policy = 0;
  uint64_t budget = 0;
  int max_inflight = 0, max_tables = 0, ppt = 2, tile_pairs = 512, tick_item_cap = 0;
  sc_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  std::vector<ServeClass> classes;  // degree classes 2, 4, 7
  cudaEvent_t fork = nullptr;
  TickSlot slots[kSlots];
  int next_slot = 0;
  std::deque<int> slots_in_flight;
  uint32_t* stage_host = nullptr;  // pinned [max_inflight][stage_words] result staging
  ExprDev* expr_host = nullptr;    // pinned [max_inflight] expression staging
  BatchRound* rounds_host = nullptr;  // pinned [max_inflight][kMaxRounds] (large requests)
  std::vector<cudaEvent_t> stage_events;  // per staging slot: a large request's completion
  // large-proof lane: a low-priority stream of its own, with a context for table generation
  cudaStream_t lane = nullptr;
  sc_ctx* lane_ctx = nullptr;
  std::deque<ServeRequest*> lane_inflight;
  int64_t large_items = 1;         // round-0 tiles above which a request takes the lane
  size_t stage_words = 0;
  std::vector<int> free_stage;
  int64_t wave_items = 1;          // resident blocks of the largest class grid: one wave
  int64_t tick_budget = 1;         // items per tick for the larger rounds
  // shared with callers
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<ServeRequest*> incoming;
  std::unordered_map<uint64_t, std::unique_ptr<ServeRequest>> reqs;
  uint64_t next_id = 1;
  uint64_t open_requests = 0;      // submitted and not yet completed or failed
  uint64_t suspend_epoch = 0;      // sc_server_suspend calls; the worker scans its queue when it moved
  uint64_t seen_epoch = 0;
  bool stop = false;
  sc_server_stats stats{};
  // worker only
  std::deque<ServeRequest*> waiting;
  std::vector<ServeRequest*> active;
  size_t admitted_bytes = 0;
  double busy_since = -1;
  std::thread worker;
  Clock::time_point t0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  // worker-side accumulators, folded into stats under the lock
  void add_time(double sc_server_stats::*field, double dt) {
    std::lock_guard<std::mutex> lk(mu);
    stats.*field += dt;
  }
};

namespace {

int build_expr(const sc_server* S, const sc_expr& ex, ExprDev& E) {
  std::memset(&E, 0, sizeof(E));
  switch (S->L) {
    case 1: build_expr_dev<1>(ex, *S->field, E); break;
    case 2: build_expr_dev<2>(ex, *S->field, E); break;
    case 4: build_expr_dev<4>(ex, *S->field, E); break;
    default: build_expr_dev<8>(ex, *S->field, E); break;
  }
  return SC_OK;
}

// Round t of request R as the kernel's RoundArgs (buffers: tables, then fold ping-pong).
void round_args(const sc_server* S, const ServeRequest& R, int t, RoundArgs& A) {
  std::memset(&A, 0, sizeof(A));
  const int n = R.n;
  const uint64_t N = uint64_t{1} << n;
  A.round = t;
  A.num_rounds = n;
  A.mode = R.mode;
  A.fc = S->field->dev;
  A.pairs = N >> (t + 1);
  A.skip1 = (t >= 1 && A.pairs >= kServeSkip1MinPairs) ? 1 : 0;
  A.want_claim = (t + 1 < n && (N >> (t + 2)) >= kServeSkip1MinPairs) ? 1 : 0;
  if (t == 0) {
    A.fold = 0;
    A.src = R.tables;
    A.src_len = N;
  } else {
    A.fold = 1;
    A.src_len = N >> (t - 1);
    A.src = t == 1 ? R.tables : ((t & 1) ? R.fold_b : R.fold_a);
    A.dst = (t & 1) ? R.fold_a : R.fold_b;
  }
  uint32_t* s = R.state;
  const StateOffsets& o = R.so;
  A.st.counter = s + o.counter;
  A.st.status = s + o.status;
  A.st.checksum = reinterpret_cast<uint64_t*>(s + o.checksum);
  A.st.polys = s + o.polys;
  A.st.chals = s + o.chals;
  A.st.finals = s + o.finals;
  A.st.claim0 = s + o.claim0;
  A.st.claim = s + o.claim;
}

// Worker-side completion: results into the request, status published under the lock.
void publish(sc_server* S, ServeRequest* R, int status, double t_done) {
  std::lock_guard<std::mutex> lk(S->mu);
  R->status = status;
  R->t_done = t_done;
  if (status == SC_OK)
    ++S->stats.completed;
  else if (status == SC_SUSPENDED)
    ++S->stats.suspended;
  else
    ++S->stats.failed;
  --S->open_requests;
  S->cv_done.notify_all();
}

void extract_results(sc_server* S, ServeRequest* R, const uint32_t* hs) {
  const int L = S->L, n = R->n, d = R->d, K = R->K;
  R->polys.resize(static_cast<size_t>(n) * (d + 1) * L);
  for (int j = 0; j < n; ++j)
    std::memcpy(R->polys.data() + static_cast<size_t>(j) * (d + 1) * L, hs + R->so.polys + static_cast<size_t>(j) * kMaxPoints * L,
                static_cast<size_t>(d + 1) * L * 4);
  R->chals.assign(hs + R->so.chals, hs + R->so.chals + static_cast<size_t>(n) * L);
  R->finals.assign(hs + R->so.finals, hs + R->so.finals + static_cast<size_t>(1 + K) * L);
  R->claim0.assign(hs + R->so.claim0, hs + R->so.claim0 + L);
  std::memcpy(&R->checksum, hs + R->so.checksum, 8);
}

void mark_busy(sc_server* S) {
  if (S->busy_since < 0) S->busy_since = S->now();
}

void mark_idle_if_done(sc_server* S) {
  if (S->busy_since >= 0 && S->active.empty() && S->slots_in_flight.empty() && S->lane_inflight.empty()) {
    const double t = S->now();
    std::lock_guard<std::mutex> lk(S->mu);
    S->stats.busy_s += t - S->busy_since;
    S->busy_since = -1;
  }
}

// Retires finished ticks, oldest first. block: wait for the oldest one.
int retire_ticks(sc_server* S, bool block) {
  while (!S->slots_in_flight.empty()) {
    TickSlot& T = S->slots[S->slots_in_flight.front()];
    if (block) {
      const double w0 = S->now();
      SC_CUDA(cudaEventSynchronize(T.done));
      S->add_time(&sc_server_stats::wait_s, S->now() - w0);
      block = false;
    } else {
      const cudaError_t q = cudaEventQuery(T.done);
      if (q == cudaErrorNotReady) break;
      if (q != cudaSuccess) return fail(SC_ERR_CUDA, "tick: %s", cudaGetErrorString(q));
    }
    const double t = S->now();
    for (ServeRequest* R : T.completing) {
      const uint32_t* hs = S->stage_host + static_cast<size_t>(R->slot) * S->stage_words;
      const uint32_t dev_status = hs[R->so.status];
      if (R->suspending && !dev_status) {
        R->suspended_state.assign(hs, hs + R->so.total_words);
        R->suspended_done = R->round;
      } else {
        extract_results(S, R, hs);
      }
      S->free_stage.push_back(R->slot);
      R->slot = -1;
      publish(S, R, dev_status ? SC_ERR_DEVICE : (R->suspending ? SC_SUSPENDED : SC_OK), t);
    }
    T.completing.clear();
    T.busy = false;
    S->slots_in_flight.pop_front();
  }
  // the large-proof lane completes in admission order
  while (!S->lane_inflight.empty()) {
    ServeRequest* R = S->lane_inflight.front();
    const cudaError_t q = cudaEventQuery(S->stage_events[R->slot]);
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) return fail(SC_ERR_CUDA, "large request: %s", cudaGetErrorString(q));
    const double t = S->now();
    const uint32_t* hs = S->stage_host + static_cast<size_t>(R->slot) * S->stage_words;
    const uint32_t dev_status = hs[R->so.status];
    extract_results(S, R, hs);
    S->free_stage.push_back(R->slot);
    R->slot = -1;
    S->admitted_bytes -= R->footprint;  // its block went back to the pool before the event
    S->lane_inflight.pop_front();
    publish(S, R, dev_status ? SC_ERR_DEVICE : SC_OK, t);
  }
  mark_idle_if_done(S);
  return SC_OK;
}

// A large request, whole, on the lane: state, descriptors, tables, one launch per round (one
// block per tile, so the small requests' higher-priority launches take SMs as these blocks
// retire), result copy, free, completion event -- all ordered on the lane.
int issue_large(sc_server* S, ServeRequest* R) {
  if (R->first)
    SC_CUDA(cudaMemcpyAsync(R->state, R->resume_state.data(), R->so.total_words * 4, cudaMemcpyHostToDevice, S->lane));
  else
    SC_CUDA(cudaMemsetAsync(R->state, 0, R->so.total_words * 4, S->lane));
  ExprDev& E = S->expr_host[R->slot];
  build_expr(S, R->expr, E);
  SC_CUDA(cudaMemcpyAsync(R->expr_dev, &E, sizeof(ExprDev), cudaMemcpyHostToDevice, S->lane));
  BatchRound* rh = S->rounds_host + static_cast<size_t>(R->slot) * kMaxRounds;
  int c = 0;
  while (S->classes[c].dclass != R->dclass) ++c;
  const ServeClass& C = S->classes[c];
  // A round's tile: the base tile, or larger so that the round is about kLaneWaves waves of
  // blocks (fewer blocks, less per-block reduction and launch work; the small requests'
  // blocks still find SMs within microseconds, as hundreds of lane blocks retire in turn).
  // Measured on B200 over 4,000 requests of the served stream at 80% load (p50 / p90 / p99 ms):
  // 1 wave 1.41 / 12.3 / 38.3, 2 waves 1.33 / 13.0 / 39.3, 4 waves 1.29-1.32 / 14.0-14.2 /
  // 41.5-45.6, 8 waves 1.22 / 14.7 / 43.5, 16 waves 1.13 / 16.0 / 46.6: more, smaller lane
  // blocks let the small requests in sooner and slow the large ones.
#ifndef SC_LANE_WAVES
#define SC_LANE_WAVES 2
#endif
  constexpr uint64_t kLaneWaves = SC_LANE_WAVES;
  std::vector<uint64_t> tiles(R->n);
  int last = R->n;  // rounds [first, last) are launched; a tail covers the rest
  for (int t = R->first; t < last; ++t) {
    BatchRound& B = rh[t];
    std::memset(&B, 0, sizeof(B));
    round_args(S, *R, t, B.args);
    const uint64_t want = B.args.pairs / (kLaneWaves * static_cast<uint64_t>(S->wave_items));
    const uint64_t thr = static_cast<uint64_t>(C.threads);
    const uint64_t tile = std::max<uint64_t>(S->tile_pairs, (want + thr - 1) / thr * thr);
    tiles[t] = tile;
    const uint64_t items = (B.args.pairs + tile - 1) / tile;
    B.expr = R->expr_dev;
    B.partials = R->partials;
    B.first_item = 0;
    B.num_items = static_cast<int32_t>(items);
    B.item_base = 0;
    B.round_items = static_cast<int32_t>(items);
    if (kServeTails && items == 1 && t + 1 < R->n) {
      set_tail(B, B.args, R->fold_a, R->fold_b);
      last = t + 1;
    }
  }
  SC_CUDA(cudaMemcpyAsync(R->rounds_dev + R->first, rh + R->first,
                          static_cast<size_t>(last - R->first) * sizeof(BatchRound), cudaMemcpyHostToDevice, S->lane));
  int rc = sc_tables_generate(S->lane_ctx, S->field, R->K, R->n, R->kinds.data(), R->seed, R->tables);
  if (!rc)
    rc = resume_folds(S->field, R->n, R->K, R->tables, R->fold_a, R->fold_b, R->state + R->so.chals, R->first,
                      S->lane_ctx->sm_count, S->lane);
  if (rc) return rc;
  for (int t = R->first; t < last; ++t) {
    BatchTickArgs A;
    A.rounds = R->rounds_dev + t;
    A.items = nullptr;
    A.num_items = rh[t].num_items;
    A.pad = 0;
    A.head = nullptr;
    A.tile = tiles[t];
    rc = batch_kernel_launch(S->L, S->kind, C.dclass, S->field, static_cast<unsigned>(A.num_items), C.threads, C.smem,
                             S->lane, A);
    if (rc) return rc;
  }
  SC_CUDA(cudaMemcpyAsync(S->stage_host + static_cast<size_t>(R->slot) * S->stage_words, R->state,
                          R->so.total_words * 4, cudaMemcpyDeviceToHost, S->lane));
  SC_CUDA(cudaFreeAsync(R->block, S->lane));
  R->block = nullptr;
  SC_CUDA(cudaEventRecord(S->stage_events[R->slot], S->lane));
  S->lane_inflight.push_back(R);
  return SC_OK;
}

// Queued requests marked for suspension leave where they stand: the state they were
// submitted with (zeros, or the transcript they resume).
void suspend_waiting(sc_server* S) {
  for (auto it = S->waiting.begin(); it != S->waiting.end();) {
    ServeRequest* R = *it;
    if (!R->suspend.load()) {
      ++it;
      continue;
    }
    it = S->waiting.erase(it);
    if (R->first)
      R->suspended_state = R->resume_state;
    else
      R->suspended_state.assign(R->so.total_words, 0u);
    R->suspended_done = R->first;
    R->suspending = true;
    publish(S, R, SC_SUSPENDED, S->now());
  }
}

int admit(sc_server* S) {
  while (!S->waiting.empty() && static_cast<int>(S->active.size() + S->lane_inflight.size()) < S->max_inflight &&
         !S->free_stage.empty()) {
    ServeRequest* R = S->waiting.front();
    if (S->admitted_bytes + R->footprint > S->budget) break;  // arrival order: no overtaking
    S->waiting.pop_front();
    const BlockLayout b = block_layout(R->n, R->K, S->L, S->tile_pairs);
    const uint64_t items0 = (((uint64_t{1} << R->n) >> (R->first + 1)) + S->tile_pairs - 1) / S->tile_pairs;
    R->large = static_cast<int64_t>(items0) > S->large_items;
    cudaStream_t st = R->large ? S->lane : S->stream;
    void* p = nullptr;
    const double a0 = S->now();
    const cudaError_t e = cudaMallocFromPoolAsync(&p, b.total, S->pool, st);
    S->add_time(&sc_server_stats::alloc_s, S->now() - a0);
    if (e != cudaSuccess) {
      cudaGetLastError();
      publish(S, R, SC_ERR_NOMEM, S->now());
      continue;
    }
    R->block = static_cast<char*>(p);
    R->state = reinterpret_cast<uint32_t*>(R->block + b.state);
    R->partials = reinterpret_cast<uint32_t*>(R->block + b.partials);
    R->expr_dev = reinterpret_cast<ExprDev*>(R->block + b.expr);
    R->rounds_dev = reinterpret_cast<BatchRound*>(R->block + b.rounds);
    R->tables = reinterpret_cast<uint32_t*>(R->block + b.tables);
    R->fold_a = reinterpret_cast<uint32_t*>(R->block + b.fold_a);
    R->fold_b = reinterpret_cast<uint32_t*>(R->block + b.fold_b);
    R->slot = S->free_stage.back();
    S->free_stage.pop_back();
    R->round = R->first;
    R->issued = 0;
    R->t_admit = S->now();
    S->admitted_bytes += R->footprint;
    mark_busy(S);
    if (R->large) {
      int rc = issue_large(S, R);
      if (rc) return rc;
    } else {
      if (R->first)
        SC_CUDA(cudaMemcpyAsync(R->state, R->resume_state.data(), R->so.total_words * 4, cudaMemcpyHostToDevice,
                                S->stream));
      else
        SC_CUDA(cudaMemsetAsync(R->state, 0, R->so.total_words * 4, S->stream));
      ExprDev& E = S->expr_host[R->slot];
      build_expr(S, R->expr, E);
      SC_CUDA(cudaMemcpyAsync(R->expr_dev, &E, sizeof(ExprDev), cudaMemcpyHostToDevice, S->stream));
      int rc = sc_tables_generate(S->ctx, S->field, R->K, R->n, R->kinds.data(), R->seed, R->tables);
      if (!rc)
        rc = resume_folds(S->field, R->n, R->K, R->tables, R->fold_a, R->fold_b, R->state + R->so.chals, R->first,
                          S->ctx->sm_count, S->stream);
      if (rc) return rc;
      S->active.push_back(R);
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->stats.peak_inflight = std::max<uint64_t>(S->stats.peak_inflight, S->active.size() + S->lane_inflight.size());
    S->stats.peak_footprint = std::max<uint64_t>(S->stats.peak_footprint, S->admitted_bytes);
  }
  return SC_OK;
}

// One tick over the in-flight requests. Returns SC_OK; *issued = whether anything ran.
int issue_tick(sc_server* S, bool* issued) {
  *issued = false;
  if (S->active.empty()) return SC_OK;
  const int si = S->next_slot;
  TickSlot& T = S->slots[si];
  if (T.busy) {  // the ring is full: wait for the oldest tick (it is this slot's)
    int rc = retire_ticks(S, true);
    if (rc) return rc;
  }
  const double b0 = S->now();
  // requests marked for suspension whose current round has not started leave with this tick
  std::vector<ServeRequest*> suspend_now;
  for (ServeRequest* R : S->active)
    if (R->issued == 0 && R->suspend.load()) suspend_now.push_back(R);
  for (ServeRequest* R : suspend_now) {
    R->suspending = true;
    S->active.erase(std::find(S->active.begin(), S->active.end(), R));
  }
  const int nc = static_cast<int>(S->classes.size());
  std::vector<std::vector<BatchRound>> rounds(nc);
  std::vector<std::vector<BatchItem>> items(nc);
  std::vector<ServeRequest*> done_now;
  int total_items = 0;
  // Tick composition. Phase 1: every request whose current round has at most `small` items
  // left runs all of them (small proofs advance one round per tick whatever else runs).
  // Phase 2: the tick's remaining item budget goes to the larger rounds in admission order,
  // oldest first; the oldest always gets `small` items at least, so it advances at the
  // rate of the whole GPU and the larger proofs finish in arrival order.
  const uint64_t tile = static_cast<uint64_t>(S->tile_pairs);
  const int64_t small = std::min<int64_t>(S->wave_items, S->tick_budget);
  int64_t budget = S->tick_budget;
  auto left_items = [&](const ServeRequest* R) {
    const uint64_t pairs = (uint64_t{1} << R->n) >> (R->round + 1);
    return static_cast<int64_t>((pairs + tile - 1) / tile - R->issued);
  };
  auto add = [&](ServeRequest* R, uint64_t give) {
    int c = 0;
    while (S->classes[c].dclass != R->dclass) ++c;
    const uint64_t pairs = (uint64_t{1} << R->n) >> (R->round + 1);
    const uint64_t round_items = (pairs + tile - 1) / tile;
    BatchRound B;
    std::memset(&B, 0, sizeof(B));
    round_args(S, *R, R->round, B.args);
    B.expr = R->expr_dev;
    B.partials = R->partials;
    B.first_item = static_cast<int32_t>(items[c].size());
    B.num_items = static_cast<int32_t>(give);
    B.item_base = static_cast<int32_t>(R->issued);
    B.round_items = static_cast<int32_t>(round_items);
    const bool tail = kServeTails && round_items == 1 && R->round + 1 < R->n;
    if (tail) set_tail(B, B.args, R->fold_a, R->fold_b);
    const int32_t ridx = static_cast<int32_t>(rounds[c].size());
    for (uint64_t i = R->issued; i < R->issued + give; ++i) {
      BatchItem I;
      I.round = ridx;
      I.pad = 0;
      I.start = i * tile;
      I.count = std::min<uint64_t>(tile, pairs - i * tile);
      items[c].push_back(I);
    }
    rounds[c].push_back(B);
    total_items += static_cast<int>(give);
    R->issued += give;
    if (R->issued == round_items) {
      R->issued = 0;
      R->round = tail ? R->n : R->round + 1;
      if (R->round == R->n) done_now.push_back(R);
    }
  };
  std::vector<ServeRequest*> large;
  for (ServeRequest* R : S->active) {
    const int64_t left = left_items(R);
    if (left > small) {
      large.push_back(R);
    } else if (total_items + left <= S->tick_item_cap) {
      add(R, static_cast<uint64_t>(left));
      budget -= left;
    }
  }
  for (size_t q = 0; q < large.size(); ++q) {
    ServeRequest* R = large[q];
    int64_t give = std::min<int64_t>(left_items(R), q == 0 ? std::max<int64_t>(budget, small) : budget);
    give = std::min<int64_t>(give, S->tick_item_cap - total_items);
    if (give <= 0) break;
    add(R, static_cast<uint64_t>(give));
    budget -= give;
  }
  // pack heads | per class: rounds, items into the slot's pinned buffer; one upload
  size_t off = 64;
  std::vector<size_t> r_off(nc), i_off(nc);
  for (int c = 0; c < nc; ++c) {
    r_off[c] = off = align_up(off, 16);
    off += rounds[c].size() * sizeof(BatchRound);
    i_off[c] = off = align_up(off, 16);
    off += items[c].size() * sizeof(BatchItem);
  }
  if (off > T.cap) return fail(SC_ERR_NOMEM, "tick descriptors %zu B exceed the slot's %zu B", off, T.cap);
  std::memset(T.host, 0, 64);
  for (int c = 0; c < nc; ++c) {
    if (!rounds[c].empty()) std::memcpy(T.host + r_off[c], rounds[c].data(), rounds[c].size() * sizeof(BatchRound));
    if (!items[c].empty()) std::memcpy(T.host + i_off[c], items[c].data(), items[c].size() * sizeof(BatchItem));
  }
  SC_CUDA(cudaMemcpyAsync(T.dev, T.host, off, cudaMemcpyHostToDevice, S->stream));
  SC_CUDA(cudaEventRecord(S->fork, S->stream));
  for (int c = 0; c < nc; ++c) {
    if (items[c].empty()) continue;
    ServeClass& C = S->classes[c];
    BatchTickArgs A;
    A.rounds = reinterpret_cast<const BatchRound*>(T.dev + r_off[c]);
    A.items = reinterpret_cast<const BatchItem*>(T.dev + i_off[c]);
    A.num_items = static_cast<int32_t>(items[c].size());
    A.pad = 0;
    A.head = reinterpret_cast<uint32_t*>(T.dev) + c;
    A.tile = 0;
    SC_CUDA(cudaStreamWaitEvent(C.stream, S->fork, 0));
    const unsigned grid = static_cast<unsigned>(std::min(C.grid, std::max(1, A.num_items)));
    int rc = batch_kernel_launch(S->L, S->kind, C.dclass, S->field, grid, C.threads, C.smem, C.stream, A);
    if (rc) return rc;
    SC_CUDA(cudaEventRecord(C.done, C.stream));
    SC_CUDA(cudaStreamWaitEvent(S->stream, C.done, 0));
  }
  // finished and suspended requests: state to pinned staging, block back to the pool
  for (ServeRequest* R : suspend_now) {
    SC_CUDA(cudaMemcpyAsync(S->stage_host + static_cast<size_t>(R->slot) * S->stage_words, R->state,
                            R->so.total_words * 4, cudaMemcpyDeviceToHost, S->stream));
    SC_CUDA(cudaFreeAsync(R->block, S->stream));
    R->block = nullptr;
    S->admitted_bytes -= R->footprint;
    T.completing.push_back(R);
  }
  for (ServeRequest* R : done_now) {
    SC_CUDA(cudaMemcpyAsync(S->stage_host + static_cast<size_t>(R->slot) * S->stage_words, R->state,
                            R->so.total_words * 4, cudaMemcpyDeviceToHost, S->stream));
    SC_CUDA(cudaFreeAsync(R->block, S->stream));
    R->block = nullptr;
    S->admitted_bytes -= R->footprint;
    S->active.erase(std::find(S->active.begin(), S->active.end(), R));
    T.completing.push_back(R);
  }
  SC_CUDA(cudaEventRecord(T.done, S->stream));
  T.busy = true;
  S->slots_in_flight.push_back(si);
  S->next_slot = (si + 1) % kSlots;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    ++S->stats.ticks;
    S->stats.items += static_cast<uint64_t>(total_items);
    S->stats.build_s += S->now() - b0;
  }
  *issued = true;
  return SC_OK;
}

// Fails every request the worker holds (after a CUDA error the stream is unusable).
void fail_all(sc_server* S, int rc) {
  const double t = S->now();
  std::vector<ServeRequest*> all(S->waiting.begin(), S->waiting.end());
  all.insert(all.end(), S->active.begin(), S->active.end());
  all.insert(all.end(), S->lane_inflight.begin(), S->lane_inflight.end());
  for (int s = 0; s < kSlots; ++s)
    for (ServeRequest* R : S->slots[s].completing) all.push_back(R);
  S->waiting.clear();
  S->active.clear();
  S->lane_inflight.clear();
  for (int s = 0; s < kSlots; ++s) S->slots[s].completing.clear();
  S->slots_in_flight.clear();
  for (ServeRequest* R : all) publish(S, R, rc, t);
}

void loop_continuous(sc_server* S) {
  bool lane_only = false;  // last pass: nothing to issue, only the lane in flight
  bool scan_waiting = false;  // a suspension was asked for since the last pass
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      const bool idle = S->waiting.empty() && S->active.empty() && S->slots_in_flight.empty() && S->lane_inflight.empty();
      if (idle) {
        S->cv_work.wait(lk, [S] { return S->stop || !S->incoming.empty(); });
      } else if (lane_only) {
        // poll the lane's completions, waking early for a new request
        const double w0 = S->now();
        S->cv_work.wait_for(lk, std::chrono::microseconds(100), [S] { return S->stop || !S->incoming.empty(); });
        S->stats.wait_s += S->now() - w0;
      }
      scan_waiting = S->suspend_epoch != S->seen_epoch;
      S->seen_epoch = S->suspend_epoch;
      while (!S->incoming.empty()) {
        S->waiting.push_back(S->incoming.front());
        S->incoming.pop_front();
      }
      if (S->stop && S->waiting.empty() && S->active.empty() && S->slots_in_flight.empty() && S->lane_inflight.empty())
        return;
    }
    int rc = retire_ticks(S, false);
    if (scan_waiting) suspend_waiting(S);
    if (!rc) rc = admit(S);
    bool issued = false;
    if (!rc) rc = issue_tick(S, &issued);
    lane_only = false;
    if (!rc && !issued) {
      if (!S->slots_in_flight.empty())
        rc = retire_ticks(S, true);
      else
        lane_only = !S->lane_inflight.empty();
    }
    if (rc) {
      fail_all(S, rc);
      cudaStreamSynchronize(S->stream);
      cudaStreamSynchronize(S->lane);
      cudaGetLastError();
    }
  }
}

void loop_fifo(sc_server* S) {
  for (;;) {
    ServeRequest* R = nullptr;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [S] { return S->stop || !S->incoming.empty(); });
      if (S->incoming.empty()) return;  // stop with nothing queued
      R = S->incoming.front();
      S->incoming.pop_front();
    }
    if (R->suspend.load()) {  // not started: leaves as submitted
      R->suspended_state = R->first ? R->resume_state : std::vector<uint32_t>(R->so.total_words, 0u);
      R->suspended_done = R->first;
      R->suspending = true;
      publish(S, R, SC_SUSPENDED, S->now());
      continue;
    }
    R->t_admit = S->now();
    mark_busy(S);
    const uint64_t N = uint64_t{1} << R->n;
    void* p = nullptr;
    int rc = SC_OK;
    cudaError_t e = cudaMallocFromPoolAsync(&p, static_cast<size_t>(R->K) * S->L * N * 4, S->pool, S->stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      rc = fail(SC_ERR_NOMEM, "table allocation: %s", cudaGetErrorString(e));
    }
    if (!rc) rc = sc_tables_generate(S->ctx, S->field, R->K, R->n, R->kinds.data(), R->seed, static_cast<uint32_t*>(p));
    if (!rc) {
      const int L = S->L;
      R->polys.resize(static_cast<size_t>(R->n) * (R->d + 1) * L);
      R->chals.resize(static_cast<size_t>(R->n) * L);
      R->finals.resize(static_cast<size_t>(1 + R->K) * L);
      R->claim0.resize(L);
      if (R->first) {  // resumed: the rest of the proof from its transcript's state
        std::vector<uint32_t> st = R->resume_state;
        rc = prove_segment(S->ctx, S->field, &R->expr, R->n, static_cast<const uint32_t*>(p), R->mode, nullptr,
                           R->first, R->n, st.data());
        if (!rc) extract_results(S, R, st.data());
      } else {
        rc = sc_prove(S->ctx, S->field, &R->expr, R->n, static_cast<const uint32_t*>(p), R->mode, nullptr,
                      R->polys.data(), R->chals.data(), R->finals.data(), R->claim0.data(), &R->checksum);
      }
    }
    if (p) cudaFreeAsync(p, S->stream);
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->stats.peak_inflight = std::max<uint64_t>(S->stats.peak_inflight, 1);
      S->stats.peak_footprint = std::max<uint64_t>(S->stats.peak_footprint, R->footprint);
    }
    publish(S, R, rc, S->now());
    const double t = S->now();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->stats.busy_s += t - S->busy_since;
    }
    S->busy_since = -1;
  }
}

void worker_main(sc_server* S) {
  cudaSetDevice(S->device);
  if (S->policy == SC_SERVE_FIFO_PLAIN)
    loop_fifo(S);
  else
    loop_continuous(S);
}

size_t request_footprint(const sc_server* S, int n, int K) {
  if (S->policy == SC_SERVE_FIFO_PLAIN) return align_up(static_cast<size_t>(K) * S->L * (size_t{1} << n) * 4, kAlign);
  return block_layout(n, K, S->L, S->tile_pairs).total;
}

int check_request(const sc_server* S, const sc_expr* expr, int num_rounds) {
  if (!expr) return fail(SC_ERR_INVALID, "NULL expression");
  if (num_rounds < 1 || num_rounds > kMaxRounds) return fail(SC_ERR_INVALID, "num_rounds %d outside 1..%d", num_rounds, kMaxRounds);
  if (expr->num_vars > S->max_tables)
    return fail(SC_ERR_UNSUPPORTED, "expression has %d tables; this server takes at most %d", expr->num_vars, S->max_tables);
  return SC_OK;
}

void destroy_resources(sc_server* S) {
  cudaSetDevice(S->device);
  if (S->stream) cudaStreamSynchronize(S->stream);
  for (ServeClass& C : S->classes) {
    if (C.stream) cudaStreamSynchronize(C.stream);
    if (C.done) cudaEventDestroy(C.done);
    if (C.stream) cudaStreamDestroy(C.stream);
  }
  for (TickSlot& T : S->slots) {
    if (T.host) cudaFreeHost(T.host);
    if (T.dev) cudaFree(T.dev);
    if (T.done) cudaEventDestroy(T.done);
  }
  if (S->lane) cudaStreamSynchronize(S->lane);
  if (S->fork) cudaEventDestroy(S->fork);
  for (cudaEvent_t e : S->stage_events) cudaEventDestroy(e);
  if (S->stage_host) cudaFreeHost(S->stage_host);
  if (S->expr_host) cudaFreeHost(S->expr_host);
  if (S->rounds_host) cudaFreeHost(S->rounds_host);
  if (S->ctx) sc_ctx_destroy(S->ctx);
  if (S->lane_ctx) sc_ctx_destroy(S->lane_ctx);
  if (S->pool) cudaMemPoolDestroy(S->pool);
  if (S->stream) cudaStreamDestroy(S->stream);
  if (S->lane) cudaStreamDestroy(S->lane);
}

}  // namespace

extern "C" {

int sc_server_create(int device, const sc_field* field, int policy, uint64_t hbm_budget_bytes, int max_inflight,
                     int max_tables, int threads, int pairs_per_thread, int chunk_items, sc_server** out) {
  if (!field || !out) return fail(SC_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (policy != SC_SERVE_CONTINUOUS && policy != SC_SERVE_FIFO_PLAIN) return fail(SC_ERR_INVALID, "unknown policy %d", policy);
  if (hbm_budget_bytes == 0) return fail(SC_ERR_INVALID, "zero HBM budget");
  if (max_inflight < 1 || max_inflight > 4096) return fail(SC_ERR_INVALID, "max_inflight %d outside 1..4096", max_inflight);
  if (max_tables < 1 || max_tables > kMaxVars) return fail(SC_ERR_INVALID, "max_tables %d outside 1..%d", max_tables, kMaxVars);
  if (threads != 0 && (threads < 32 || threads > 256 || threads % 32))
    return fail(SC_ERR_INVALID, "threads must be 0 (auto) or a multiple of 32 in 32..256");
  if (pairs_per_thread < 0 || pairs_per_thread > 64) return fail(SC_ERR_INVALID, "pairs_per_thread outside 0..64");
  if (chunk_items < 0) return fail(SC_ERR_INVALID, "chunk_items < 0");
  if (field->device != device) return fail(SC_ERR_INVALID, "field lives on device %d, not %d", field->device, device);
  SC_CUDA(cudaSetDevice(device));
  std::unique_ptr<sc_server> S(new (std::nothrow) sc_server());
  if (!S) return fail(SC_ERR_NOMEM, "host allocation failed");
  S->device = device;
  S->field = field;
  S->L = field->hf.L;
  S->kind = field_kind(field->hf.p, S->L);
  S->policy = policy;
  S->budget = hbm_budget_bytes;
  S->max_inflight = max_inflight;
  S->max_tables = max_tables;
  // default tile: 1 pair a thread. Measured on B200 over 4,000 requests of the served stream
  // at 80% load, 4-limb kernels at 2 blocks/SM (p50 / p90 / p99 ms): 1 pair 0.99 / 7.6 / 25.0,
  // 2 pairs 1.12 / 7.15 / 25.0, 4 pairs 1.40 / 7.15 / 26.1. The tick budget (chunk_items,
  // 0.5-4 waves) changed p50 by under 2%.
  S->ppt = pairs_per_thread ? pairs_per_thread : 1;
  S->stats.budget = hbm_budget_bytes;
  S->t0 = Clock::now();
  auto bail = [&](int rc) {
    destroy_resources(S.get());
    return rc;
  };
  // priorities: the small requests' ticks above the large-proof lane
  int prio_low = 0, prio_high = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&S->stream, cudaStreamNonBlocking, prio_high);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&S->lane, cudaStreamNonBlocking, prio_low);
  if (e != cudaSuccess) return bail(fail(SC_ERR_CUDA, "stream: %s", cudaGetErrorString(e)));
  int rc = sc_ctx_create(device, S->stream, &S->ctx);
  if (!rc) rc = sc_ctx_create(device, S->lane, &S->lane_ctx);
  if (rc) return bail(rc);
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  e = cudaMemPoolCreate(&S->pool, &props);
  if (e != cudaSuccess) return bail(fail(SC_ERR_CUDA, "memory pool: %s", cudaGetErrorString(e)));
  uint64_t keep = ~uint64_t{0};  // freed blocks stay mapped in the pool for the next request
  e = cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  // a block freed on the lane is reused by the other stream only once its free completed:
  // no dependency that would hold small requests behind the lane
  int no = 0;
  if (e == cudaSuccess) e = cudaMemPoolSetAttribute(S->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
  if (e != cudaSuccess) return bail(fail(SC_ERR_CUDA, "memory pool attribute: %s", cudaGetErrorString(e)));
  // one tile size for every class (a request's partial slots are sized by it)
  int cls_threads = kernel_threads(S->L);
  if (threads) cls_threads = std::min(threads, cls_threads);
  const int per_thread = round_smem_words_per_thread(max_tables, S->L) * 4;
  while (cls_threads > 32 && static_cast<size_t>(cls_threads) * per_thread > static_cast<size_t>(kMaxDynSmem)) cls_threads -= 32;
  S->tile_pairs = cls_threads * S->ppt;
  int max_grid = 1;
  for (int dc : {2, 4, 7}) {
    ServeClass C;
    C.dclass = dc;
    if ((rc = batch_kernel_setup(S->L, S->kind, dc, max_tables, cls_threads, S->ctx->sm_count, &C.threads, &C.grid,
                                 &C.smem)))
      return bail(rc);
    max_grid = std::max(max_grid, C.grid);
    e = cudaStreamCreateWithPriority(&C.stream, cudaStreamNonBlocking, prio_high);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&C.done, cudaEventDisableTiming);
    S->classes.push_back(C);
    if (e != cudaSuccess) return bail(fail(SC_ERR_CUDA, "class stream: %s", cudaGetErrorString(e)));
  }
  S->wave_items = max_grid;
  S->large_items = max_grid;
  S->tick_budget = chunk_items ? chunk_items : 2 * max_grid;
  S->tick_item_cap = static_cast<int>(std::max<int64_t>(8 * max_grid, 2 * S->tick_budget));
  e = cudaEventCreateWithFlags(&S->fork, cudaEventDisableTiming);
  if (e != cudaSuccess) return bail(fail(SC_ERR_CUDA, "event: %s", cudaGetErrorString(e)));
  const size_t slot_cap = 64 + 3 * 2 * 16 + static_cast<size_t>(max_inflight) * sizeof(BatchRound) +
                          static_cast<size_t>(S->tick_item_cap) * sizeof(BatchItem);
  for (TickSlot& T : S->slots) {
    T.cap = slot_cap;
    e = cudaMallocHost(&T.host, slot_cap);
    if (e == cudaSuccess) e = cudaMalloc(&T.dev, slot_cap);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&T.done, cudaEventDisableTiming);
    if (e != cudaSuccess) return bail(fail(SC_ERR_NOMEM, "tick slot: %s", cudaGetErrorString(e)));
  }
  S->stage_words = align_up(state_offsets(kMaxRounds, max_tables, S->L).total_words, 64);
  e = cudaMallocHost(&S->stage_host, static_cast<size_t>(max_inflight) * S->stage_words * 4);
  if (e == cudaSuccess) e = cudaMallocHost(&S->expr_host, static_cast<size_t>(max_inflight) * sizeof(ExprDev));
  if (e == cudaSuccess)
    e = cudaMallocHost(&S->rounds_host, static_cast<size_t>(max_inflight) * kMaxRounds * sizeof(BatchRound));
  for (int i = 0; e == cudaSuccess && i < max_inflight; ++i) {
    cudaEvent_t ev;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) S->stage_events.push_back(ev);
  }
  if (e != cudaSuccess) return bail(fail(SC_ERR_NOMEM, "pinned staging: %s", cudaGetErrorString(e)));
  for (int i = max_inflight - 1; i >= 0; --i) S->free_stage.push_back(i);
  sc_server* raw = S.release();
  raw->worker = std::thread(worker_main, raw);
  *out = raw;
  return SC_OK;
}

int sc_server_reserve(sc_server* S, uint64_t bytes) {
  if (!S) return fail(SC_ERR_INVALID, "NULL server");
  if (bytes == 0) return SC_OK;
  // on the caller's thread, on a stream of its own: the pool is thread-safe
  SC_CUDA(cudaSetDevice(S->device));
  cudaStream_t s = nullptr;
  SC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, S->pool, s);
  if (e == cudaSuccess) e = cudaFreeAsync(p, s);
  const cudaError_t e2 = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return fail(SC_ERR_NOMEM, "reserving %llu B: %s", static_cast<unsigned long long>(bytes), cudaGetErrorString(e));
  if (e2 != cudaSuccess) return fail(SC_ERR_CUDA, "reserve: %s", cudaGetErrorString(e2));
  return SC_OK;
}

int sc_server_footprint(const sc_server* S, const sc_expr* expr, int num_rounds, uint64_t* out_bytes) {
  if (!S || !out_bytes) return fail(SC_ERR_INVALID, "NULL argument");
  int rc = check_request(S, expr, num_rounds);
  if (rc) return rc;
  *out_bytes = request_footprint(S, num_rounds, expr->num_vars);
  if (*out_bytes > S->budget)
    return fail(SC_ERR_UNSUPPORTED, "footprint %llu B exceeds the HBM budget %llu B",
                static_cast<unsigned long long>(*out_bytes), static_cast<unsigned long long>(S->budget));
  return SC_OK;
}

}  // extern "C"

namespace {

// Queues a request; `resume` (state words) and `first` continue a transcript.
int submit_request(sc_server* S, const sc_expr* expr, int num_rounds, const int32_t* table_kinds, uint64_t seed,
                   int challenge_mode, int first, const uint32_t* resume, uint64_t* out_id) {
  if (!S || !expr || !table_kinds || !out_id) return fail(SC_ERR_INVALID, "NULL argument");
  if (challenge_mode != SC_CHALLENGE_SHA3 && challenge_mode != SC_CHALLENGE_FIXED)
    return fail(SC_ERR_INVALID, "served proofs derive their challenges: SHA3 or fixed mode");
  uint64_t fp = 0;
  int rc = sc_server_footprint(S, expr, num_rounds, &fp);
  if (rc) return rc;
  for (int k = 0; k < expr->num_vars; ++k)
    if (table_kinds[k] < 0) return fail(SC_ERR_INVALID, "table_kinds[%d] = %d", k, table_kinds[k]);
  std::unique_ptr<ServeRequest> R(new (std::nothrow) ServeRequest());
  if (!R) return fail(SC_ERR_NOMEM, "host allocation failed");
  R->expr = *expr;
  R->n = num_rounds;
  R->K = expr->num_vars;
  R->d = expr->degree;
  R->dclass = degree_class(expr->degree);
  R->kinds.assign(table_kinds, table_kinds + expr->num_vars);
  R->seed = seed;
  R->mode = challenge_mode;
  R->footprint = fp;
  R->so = state_offsets(num_rounds, R->K, S->L);
  R->first = first;
  if (first) R->resume_state.assign(resume, resume + R->so.total_words);
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) return fail(SC_ERR_INVALID, "server is shutting down");
  R->id = S->next_id++;
  R->t_submit = S->now();
  *out_id = R->id;
  S->incoming.push_back(R.get());
  S->reqs.emplace(R->id, std::move(R));
  ++S->stats.submitted;
  ++S->open_requests;
  S->cv_work.notify_one();
  return SC_OK;
}

}  // namespace

extern "C" {

int sc_server_submit(sc_server* S, const sc_expr* expr, int num_rounds, const int32_t* table_kinds, uint64_t seed,
                     int challenge_mode, uint64_t* out_id) {
  return submit_request(S, expr, num_rounds, table_kinds, seed, challenge_mode, 0, nullptr, out_id);
}

int sc_server_submit_resume(sc_server* S, const sc_expr* expr, const int32_t* table_kinds, uint64_t seed,
                            const uint32_t* transcript, uint64_t words, uint64_t* out_id) {
  if (!S || !expr || !table_kinds || !out_id) return fail(SC_ERR_INVALID, "NULL argument");
  TranscriptInfo I;
  int rc = transcript_parse(transcript, words, &I);
  if (!rc) rc = transcript_match(I, S->field->hf, *expr);
  if (rc) return rc;
  if (I.done == I.n) return fail(SC_ERR_INVALID, "the transcript's proof is complete");
  if (I.tag != seeded_tables_tag(expr->num_vars, table_kinds, seed))
    return fail(SC_ERR_INVALID, "the transcript is of other tables (table kinds or seed differ)");
  const uint32_t* state = transcript + kTranscriptHeader;
  const StateOffsets so = state_offsets(I.n, I.K, I.L);
  if (state[so.counter] || state[so.status]) return fail(SC_ERR_INVALID, "transcript state records a device error");
  return submit_request(S, expr, I.n, table_kinds, seed, I.mode, I.done, state, out_id);
}

int sc_server_suspend(sc_server* S, uint64_t id) {
  if (!S) return fail(SC_ERR_INVALID, "NULL server");
  std::lock_guard<std::mutex> lk(S->mu);
  if (id == 0) {
    for (auto& kv : S->reqs)
      if (kv.second->status == SC_ERR_PENDING) kv.second->suspend.store(true);
  } else {
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return fail(SC_ERR_INVALID, "unknown request %llu", static_cast<unsigned long long>(id));
    it->second->suspend.store(true);
  }
  ++S->suspend_epoch;
  S->cv_work.notify_all();
  return SC_OK;
}

int sc_server_transcript(sc_server* S, uint64_t id, uint32_t* transcript, uint64_t words) {
  if (!S || !transcript) return fail(SC_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return fail(SC_ERR_INVALID, "unknown request %llu", static_cast<unsigned long long>(id));
  const ServeRequest* R = it->second.get();
  if (R->status != SC_SUSPENDED)
    return fail(R->status == SC_ERR_PENDING ? SC_ERR_PENDING : SC_ERR_INVALID,
                "request %llu is not suspended (status %d)", static_cast<unsigned long long>(id), R->status);
  const size_t need = transcript_words(R->n, R->K, S->L);
  if (words < need)
    return fail(SC_ERR_INVALID, "transcript needs %zu words, got %llu", need, static_cast<unsigned long long>(words));
  transcript_header(transcript, S->field->hf, R->expr, R->n, R->mode, R->suspended_done,
                    seeded_tables_tag(R->K, R->kinds.data(), R->seed));
  std::memcpy(transcript + kTranscriptHeader, R->suspended_state.data(), R->suspended_state.size() * 4);
  return SC_OK;
}

int sc_server_wait(sc_server* S, uint64_t id, int timeout_ms) {
  if (!S) return fail(SC_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return fail(SC_ERR_INVALID, "unknown request %llu", static_cast<unsigned long long>(id));
  ServeRequest* R = it->second.get();
  auto ready = [R] { return R->status != SC_ERR_PENDING; };
  if (timeout_ms < 0)
    S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return fail(SC_ERR_TIMEOUT, "request %llu not done after %d ms", static_cast<unsigned long long>(id), timeout_ms);
  if (R->status == SC_SUSPENDED) return SC_SUSPENDED;
  if (R->status != SC_OK) return fail(R->status, "request %llu failed with status %d", static_cast<unsigned long long>(id), R->status);
  return SC_OK;
}

int sc_server_drain(sc_server* S, int timeout_ms) {
  if (!S) return fail(SC_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto ready = [S] { return S->open_requests == 0; };
  if (timeout_ms < 0)
    S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return fail(SC_ERR_TIMEOUT, "%llu requests still open after %d ms", static_cast<unsigned long long>(S->open_requests), timeout_ms);
  return SC_OK;
}

int sc_server_result(sc_server* S, uint64_t id, uint32_t* out_round_polys, uint32_t* out_challenges, uint32_t* out_finals,
                     uint32_t* out_claim0, uint64_t* out_checksum) {
  if (!S) return fail(SC_ERR_INVALID, "NULL server");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return fail(SC_ERR_INVALID, "unknown request %llu", static_cast<unsigned long long>(id));
  const ServeRequest* R = it->second.get();
  if (R->status == SC_ERR_PENDING) return fail(SC_ERR_PENDING, "request %llu has not completed", static_cast<unsigned long long>(id));
  if (R->status == SC_SUSPENDED)
    return fail(SC_SUSPENDED, "request %llu was suspended: read its transcript", static_cast<unsigned long long>(id));
  if (R->status != SC_OK) return fail(R->status, "request %llu failed with status %d", static_cast<unsigned long long>(id), R->status);
  if (out_round_polys) std::memcpy(out_round_polys, R->polys.data(), R->polys.size() * 4);
  if (out_challenges) std::memcpy(out_challenges, R->chals.data(), R->chals.size() * 4);
  if (out_finals) std::memcpy(out_finals, R->finals.data(), R->finals.size() * 4);
  if (out_claim0) std::memcpy(out_claim0, R->claim0.data(), R->claim0.size() * 4);
  if (out_checksum) *out_checksum = R->checksum;
  return SC_OK;
}

int sc_server_times(sc_server* S, uint64_t id, double* out_submit_s, double* out_admit_s, double* out_done_s) {
  if (!S) return fail(SC_ERR_INVALID, "NULL server");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return fail(SC_ERR_INVALID, "unknown request %llu", static_cast<unsigned long long>(id));
  const ServeRequest* R = it->second.get();
  if (out_submit_s) *out_submit_s = R->t_submit;
  if (out_admit_s) *out_admit_s = R->status == SC_ERR_PENDING ? -1.0 : R->t_admit;
  if (out_done_s) *out_done_s = R->status == SC_ERR_PENDING ? -1.0 : R->t_done;
  return SC_OK;
}

int sc_server_release(sc_server* S, uint64_t id) {
  if (!S) return fail(SC_ERR_INVALID, "NULL server");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return fail(SC_ERR_INVALID, "unknown request %llu", static_cast<unsigned long long>(id));
  if (it->second->status == SC_ERR_PENDING)
    return fail(SC_ERR_PENDING, "request %llu has not completed", static_cast<unsigned long long>(id));
  S->reqs.erase(it);
  return SC_OK;
}

int sc_server_stats_get(sc_server* S, sc_server_stats* out) {
  if (!S || !out) return fail(SC_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->stats;
  return SC_OK;
}

int sc_server_destroy(sc_server* S) {
  if (!S) return SC_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv_work.notify_all();
  }
  if (S->worker.joinable()) S->worker.join();
  destroy_resources(S);
  delete S;
  return SC_OK;
}

}  // extern "C"
