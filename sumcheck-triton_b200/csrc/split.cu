// One proof split across ranks (GPUs): each rank holds a contiguous chunk of every table.
//
// With W = 2^w ranks and n variables, rank r holds entries [r C, (r + 1) C), C = 2^(n - w), of
// every table. The pairs of rounds 0 .. n - w - 1 lie inside a chunk, so those rounds run on
// each rank's chunk alone (fold of the previous round fused, as always) and produce the rank's
// share of g_j(0..d); the shares are exchanged (an all-gather of (d + 1) L words per rank and
// round: the host's collective, NCCL over NVLink on a GPU cluster) and every rank sums them in
// rank order and finalises the round itself -- checksum, SHA3 challenge, claim -- with the
// same device code as a whole proof, so every rank derives the same r_j and nothing is
// broadcast. After the chunk rounds each rank's chunk is folded down to one entry per table;
// those W entries (K L words per rank) are gathered, and every rank proves the last w rounds
// on the W-entry tables. Every rank ends with the same outputs, bit-identical to sc_prove on
// the whole tables.
#include "host_common.h"

using namespace sc;
using namespace sc_host;

namespace {

constexpr uint64_t kSplitSkip1MinPairs = uint64_t{1} << 12;

// Sums the ranks' shares of one round (rank order) and finalises the round (one warp).
template <int L, int K>
__global__ void split_commit_kernel(const RoundArgs A, const ExprDev E, const FieldParams<L, K> F,
                                    const uint32_t* parts, int world) {
  __shared__ __align__(16) uint32_t g_sm[kMaxPoints * kMaxLimbs];
  __shared__ __align__(16) uint8_t msg[3 * 136];
  const int lane = threadIdx.x;
  const int d = E.degree;
  if (lane <= d) {
    Fe<L> acc = fe_zero<L>();
    for (int r = 0; r < world; ++r) acc = fe_add(acc, ld_fe<L>(parts + (static_cast<size_t>(r) * (d + 1) + lane) * L), F);
    st_fe<L>(g_sm + lane * L, acc);
  }
  __syncwarp();
  finalize_round<L, K>(A, E, F, g_sm, msg);
}

}  // namespace

struct sc_split {
  sc_ctx* ctx = nullptr;
  const sc_field* field = nullptr;
  sc_expr expr;
  ExprDev E{};
  int L = 0, kind = 0, dclass = 2, d = 0, K = 0;
  int n = 0, world = 1, rank = 0, w = 0, local_rounds = 0;
  uint64_t C = 0;              // entries per table in this rank's chunk
  const uint32_t* tables = nullptr;
  int mode = SC_CHALLENGE_SHA3;
  int next = 0;                // next round to run
  bool committed = true;       // the last run round was committed
  StateOffsets so{};
  DevBuf fold_a, fold_b, partials, state, ext, parts, tail, tail_a, tail_b;
  uint32_t* host = nullptr;    // pinned staging
  size_t host_words = 0;
  int threads = 256, grid_max = 1;
  size_t smem = 0;

  uint64_t round_pairs(int j) const {
    return j < local_rounds ? (C >> (j + 1)) : ((uint64_t{1} << w) >> (j - local_rounds + 1));
  }
  bool skip1(int j) const { return j >= 1 && j < n && round_pairs(j) >= kSplitSkip1MinPairs; }
};

namespace {

// The round kernel of a split proof's rounds: the compile-time shape kernel when the host
// matched one (degree class 4), as for a whole proof; else the generic evaluator.
template <int L, int K, int D>
using SplitKern = void (*)(const RoundArgs, const ExprDev, const FieldParams<L, K>);

template <int L, int K, int D>
SplitKern<L, K, D> split_kernel(const sc_split* S) {
  if constexpr (D == 4) {
    if (S->E.shape == kShapeZerocheck) return round_kernel<L, K, 4, kShapeZerocheck>;
    if (S->E.shape == kShapeAbcg) return round_kernel<L, K, 4, kShapeAbcg>;
  }
  return round_kernel<L, K, D>;
}

template <int L, int K, int D>
struct SplitSetup {
  static int run(sc_split* S) {
    int threads = kernel_threads(L);
    if (S->E.shape != kShapeGeneric && D == 4) {
      S->smem = shape_round_smem_bytes(L, K, S->E.shape, threads);  // block_reduce scratch (+ the pair stage)
    } else {
      const int per_thread = round_smem_words_per_thread(S->K, L) * 4;
      while (threads > 32 && threads * per_thread > kMaxDynSmem) threads -= 32;
      S->smem = static_cast<size_t>(threads) * per_thread;
    }
    S->threads = threads;
    int bps = 0;
    SC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, split_kernel<L, K, D>(S), threads, S->smem));
    if (bps < 1) return fail(SC_ERR_UNSUPPORTED, "round kernel does not fit on an SM (K=%d, L=%d)", S->K, L);
    S->grid_max = bps * S->ctx->sm_count;
    return SC_OK;
  }
};

template <int L, int K, int D>
struct SplitRound {
  static int run(sc_split* S, const RoundArgs& A) {
    FieldParams<L, K> F;
    for (int l = 0; l < L; ++l) F.p[l] = S->field->hf.p[l];
    F.np = S->field->hf.np;
    const uint64_t want = (A.pairs + S->threads - 1) / S->threads;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(std::max<uint64_t>(want, 1), S->grid_max));
    split_kernel<L, K, D>(S)<<<grid, S->threads, S->smem, S->ctx->stream>>>(A, S->E, F);
    SC_CUDA(cudaGetLastError());
    return SC_OK;
  }
};

template <int L, int K, int D>
struct SplitCommit {
  static int run(sc_split* S, const RoundArgs& A) {
    FieldParams<L, K> F;
    for (int l = 0; l < L; ++l) F.p[l] = S->field->hf.p[l];
    F.np = S->field->hf.np;
    split_commit_kernel<L, K><<<1, 32, 0, S->ctx->stream>>>(A, S->E, F, static_cast<const uint32_t*>(S->parts.p),
                                                            S->world);
    SC_CUDA(cudaGetLastError());
    return SC_OK;
  }
};

// RoundArgs of round j: chunk rounds over the rank's tables and fold buffers, the last w rounds
// over the gathered tail tables.
void split_args(const sc_split* S, int j, RoundArgs& A) {
  std::memset(&A, 0, sizeof(A));
  A.round = j;
  A.num_rounds = S->n;
  A.mode = S->mode;
  A.fc = S->field->dev;
  A.partials = static_cast<uint32_t*>(S->partials.p);
  uint32_t* st = static_cast<uint32_t*>(S->state.p);
  A.st.counter = st + S->so.counter;
  A.st.status = st + S->so.status;
  A.st.checksum = reinterpret_cast<uint64_t*>(st + S->so.checksum);
  A.st.polys = st + S->so.polys;
  A.st.chals = st + S->so.chals;
  A.st.finals = st + S->so.finals;
  A.st.claim0 = st + S->so.claim0;
  A.st.claim = st + S->so.claim;
  A.pairs = S->round_pairs(j);
  A.skip1 = S->skip1(j) ? 1 : 0;
  A.want_claim = S->skip1(j + 1) ? 1 : 0;
  const bool chunk = j < S->local_rounds;
  const int j0 = chunk ? 0 : S->local_rounds;  // first round over these tables
  const int t = j - j0;
  const uint32_t* base = chunk ? S->tables : static_cast<const uint32_t*>(S->tail.p);
  uint32_t* fa = static_cast<uint32_t*>(chunk ? S->fold_a.p : S->tail_a.p);
  uint32_t* fb = static_cast<uint32_t*>(chunk ? S->fold_b.p : S->tail_b.p);
  const uint64_t len0 = chunk ? S->C : (uint64_t{1} << S->w);
  if (t == 0) {
    A.fold = 0;
    A.src = base;
    A.src_len = len0;
  } else {
    A.fold = 1;
    A.src_len = len0 >> (t - 1);
    A.src = t == 1 ? base : ((t & 1) ? fb : fa);
    A.dst = (t & 1) ? fa : fb;
  }
}

int stage(sc_split* S, size_t words) {
  if (S->host_words >= words) return SC_OK;
  if (S->host) cudaFreeHost(S->host);
  S->host = nullptr;
  S->host_words = 0;
  SC_CUDA(cudaMallocHost(&S->host, words * 4));
  S->host_words = words;
  return SC_OK;
}

}  // namespace

extern "C" {

int sc_split_create(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int num_rounds, int world, int rank,
                    const uint32_t* local_tables_dev, int challenge_mode, sc_split** out) {
  if (!ctx || !field || !expr || !local_tables_dev || !out) return fail(SC_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (world < 1 || (world & (world - 1))) return fail(SC_ERR_INVALID, "world %d is not a power of two", world);
  if (rank < 0 || rank >= world) return fail(SC_ERR_INVALID, "rank %d outside 0..%d", rank, world - 1);
  if (num_rounds < 1 || num_rounds > kMaxRounds) return fail(SC_ERR_INVALID, "num_rounds %d outside 1..%d", num_rounds, kMaxRounds);
  int w = 0;
  while ((1 << w) < world) ++w;
  if (num_rounds - w < 1) return fail(SC_ERR_INVALID, "%d rounds cannot be split over %d ranks (chunks of 1 entry)", num_rounds, world);
  if (challenge_mode != SC_CHALLENGE_SHA3 && challenge_mode != SC_CHALLENGE_FIXED)
    return fail(SC_ERR_INVALID, "split proofs derive their challenges: SHA3 or fixed mode");
  if (reinterpret_cast<uintptr_t>(local_tables_dev) % 16) return fail(SC_ERR_INVALID, "tables not 16-byte aligned");
  SC_CUDA(cudaSetDevice(ctx->device));
  sc_split* S = new (std::nothrow) sc_split();
  if (!S) return fail(SC_ERR_NOMEM, "host allocation failed");
  S->ctx = ctx;
  S->field = field;
  S->expr = *expr;
  S->L = field->hf.L;
  S->kind = field_kind(field->hf.p, S->L);
  S->d = expr->degree;
  S->dclass = degree_class(expr->degree);
  S->K = expr->num_vars;
  S->n = num_rounds;
  S->world = world;
  S->rank = rank;
  S->w = w;
  S->local_rounds = num_rounds - w;
  S->C = uint64_t{1} << S->local_rounds;
  S->tables = local_tables_dev;
  S->mode = challenge_mode;
  S->so = state_offsets(num_rounds, S->K, S->L);
  switch (S->L) {
    case 1: build_expr_dev<1>(*expr, *field, S->E); break;
    case 2: build_expr_dev<2>(*expr, *field, S->E); break;
    case 4: build_expr_dev<4>(*expr, *field, S->E); break;
    default: build_expr_dev<8>(*expr, *field, S->E); break;
  }
  const size_t KL = static_cast<size_t>(S->K) * S->L;
  const size_t W = size_t{1} << w;
  int rc = dispatch<SplitSetup>(S->L, S->kind, S->dclass, S);
  if (!rc) rc = ensure(ctx, S->fold_a, (S->local_rounds >= 2 ? KL * (S->C / 2) : 1) * 4);
  if (!rc) rc = ensure(ctx, S->fold_b, (S->local_rounds >= 3 ? KL * (S->C / 4) : 1) * 4);
  if (!rc) rc = ensure(ctx, S->partials, static_cast<size_t>(S->grid_max) * kMaxPoints * S->L * 4);
  if (!rc) rc = ensure(ctx, S->state, S->so.total_words * 4);
  if (!rc) rc = ensure(ctx, S->ext, kMaxPoints * kMaxLimbs * 4);
  if (!rc) rc = ensure(ctx, S->parts, W * kMaxPoints * kMaxLimbs * 4);
  if (!rc) rc = ensure(ctx, S->tail, KL * std::max<size_t>(W, 2) * 4);
  if (!rc) rc = ensure(ctx, S->tail_a, KL * std::max<size_t>(W / 2, 2) * 4);
  if (!rc) rc = ensure(ctx, S->tail_b, KL * std::max<size_t>(W / 4, 2) * 4);
  if (!rc) rc = stage(S, std::max<size_t>({S->so.total_words, W * KL, W * kMaxPoints * kMaxLimbs, 2 * KL + 64}));
  if (!rc) {
    const cudaError_t e = cudaMemsetAsync(S->state.p, 0, S->so.total_words * 4, ctx->stream);
    if (e != cudaSuccess) rc = fail(SC_ERR_CUDA, "state: %s", cudaGetErrorString(e));
  }
  if (rc) {
    sc_split_destroy(S);
    return rc;
  }
  *out = S;
  return SC_OK;
}

int sc_split_local_rounds(const sc_split* S) { return S ? S->local_rounds : -1; }

int sc_split_round(sc_split* S, int round, uint32_t* out_share) {
  if (!S || !out_share) return fail(SC_ERR_INVALID, "NULL argument");
  if (round != S->next || !S->committed || round >= S->local_rounds)
    return fail(SC_ERR_INVALID, "round %d out of order (next is %d, %d chunk rounds)", round, S->next, S->local_rounds);
  SC_CUDA(cudaSetDevice(S->ctx->device));
  RoundArgs A;
  split_args(S, round, A);
  A.ext_out = static_cast<uint32_t*>(S->ext.p);
  int rc = dispatch<SplitRound>(S->L, S->kind, S->dclass, S, A);
  if (rc) return rc;
  const size_t words = static_cast<size_t>(S->d + 1) * S->L;
  SC_CUDA(cudaMemcpyAsync(S->host, S->ext.p, words * 4, cudaMemcpyDeviceToHost, S->ctx->stream));
  SC_CUDA(cudaStreamSynchronize(S->ctx->stream));
  std::memcpy(out_share, S->host, words * 4);
  S->committed = false;
  return SC_OK;
}

int sc_split_commit(sc_split* S, int round, const uint32_t* shares) {
  if (!S || !shares) return fail(SC_ERR_INVALID, "NULL argument");
  if (round != S->next || S->committed) return fail(SC_ERR_INVALID, "round %d has not been run", round);
  SC_CUDA(cudaSetDevice(S->ctx->device));
  const size_t words = static_cast<size_t>(S->world) * (S->d + 1) * S->L;
  std::memcpy(S->host, shares, words * 4);
  SC_CUDA(cudaMemcpyAsync(S->parts.p, S->host, words * 4, cudaMemcpyHostToDevice, S->ctx->stream));
  RoundArgs A;
  split_args(S, round, A);
  int rc = dispatch<SplitCommit>(S->L, S->kind, S->dclass, S, A);
  if (rc) return rc;
  SC_CUDA(cudaStreamSynchronize(S->ctx->stream));  // the staging buffer is reused next
  S->committed = true;
  ++S->next;
  return SC_OK;
}

int sc_split_last_entries(sc_split* S, uint32_t* out_entries) {
  if (!S || !out_entries) return fail(SC_ERR_INVALID, "NULL argument");
  if (S->next != S->local_rounds || !S->committed) return fail(SC_ERR_INVALID, "the chunk rounds are not all committed");
  SC_CUDA(cudaSetDevice(S->ctx->device));
  const int L = S->L, K = S->K;
  // T_{lr-1}: two entries per plane (the caller's tables when lr = 1, else a fold buffer)
  const int j = S->local_rounds - 1;
  const uint32_t* src = j == 0 ? S->tables : static_cast<const uint32_t*>((j & 1) ? S->fold_a.p : S->fold_b.p);
  SC_CUDA(cudaMemcpyAsync(S->host, src, static_cast<size_t>(K) * L * 2 * 4, cudaMemcpyDeviceToHost, S->ctx->stream));
  uint32_t* st = static_cast<uint32_t*>(S->state.p);
  SC_CUDA(cudaMemcpyAsync(S->host + 2 * K * L, st + S->so.chals + static_cast<size_t>(j) * L, L * 4,
                          cudaMemcpyDeviceToHost, S->ctx->stream));
  SC_CUDA(cudaStreamSynchronize(S->ctx->stream));
  const HostField& hf = S->field->hf;
  const uint32_t* r = S->host + 2 * K * L;
  for (int k = 0; k < K; ++k) {
    uint32_t e[8], o[8], dlt[8], t[8], f[8];
    for (int l = 0; l < L; ++l) {
      e[l] = S->host[(k * L + l) * 2 + 0];
      o[l] = S->host[(k * L + l) * 2 + 1];
    }
    hf.sub(o, e, dlt);
    hf.mul(r, dlt, t);
    hf.add(e, t, f);
    for (int l = 0; l < L; ++l) out_entries[k * L + l] = f[l];
  }
  return SC_OK;
}

int sc_split_finish(sc_split* S, const uint32_t* entries) {
  if (!S) return fail(SC_ERR_INVALID, "NULL argument");
  if (S->next != S->local_rounds || !S->committed) return fail(SC_ERR_INVALID, "the chunk rounds are not all committed");
  if (S->w > 0 && !entries) return fail(SC_ERR_INVALID, "NULL entries");
  SC_CUDA(cudaSetDevice(S->ctx->device));
  const int L = S->L, K = S->K;
  const size_t W = size_t{1} << S->w;
  if (S->w > 0) {
    // the W entries (rank order) as limb-planar tables of length W
    for (size_t rr = 0; rr < W; ++rr)
      for (int k = 0; k < K; ++k)
        for (int l = 0; l < L; ++l) S->host[(static_cast<size_t>(k) * L + l) * W + rr] = entries[(rr * K + k) * L + l];
    SC_CUDA(cudaMemcpyAsync(S->tail.p, S->host, static_cast<size_t>(K) * L * W * 4, cudaMemcpyHostToDevice,
                            S->ctx->stream));
    for (int j = S->local_rounds; j < S->n; ++j) {
      RoundArgs A;
      split_args(S, j, A);
      int rc = dispatch<SplitRound>(L, S->kind, S->dclass, S, A);
      if (rc) return rc;
    }
  }
  SC_CUDA(cudaStreamSynchronize(S->ctx->stream));
  S->next = S->n;
  return SC_OK;
}

int sc_split_result(sc_split* S, uint32_t* out_round_polys, uint32_t* out_challenges, uint32_t* out_finals,
                    uint32_t* out_claim0, uint64_t* out_checksum) {
  if (!S) return fail(SC_ERR_INVALID, "NULL split");
  if (S->next != S->n) return fail(SC_ERR_INVALID, "the proof is not finished");
  SC_CUDA(cudaSetDevice(S->ctx->device));
  SC_CUDA(cudaMemcpyAsync(S->host, S->state.p, S->so.total_words * 4, cudaMemcpyDeviceToHost, S->ctx->stream));
  SC_CUDA(cudaStreamSynchronize(S->ctx->stream));
  const uint32_t* hs = S->host;
  const StateOffsets& so = S->so;
  const int L = S->L, n = S->n, d = S->d;
  if (hs[so.status]) return fail(SC_ERR_DEVICE, "device status %u", hs[so.status]);
  if (out_round_polys)
    for (int j = 0; j < n; ++j)
      std::memcpy(out_round_polys + static_cast<size_t>(j) * (d + 1) * L, hs + so.polys + static_cast<size_t>(j) * kMaxPoints * L,
                  static_cast<size_t>(d + 1) * L * 4);
  if (out_challenges) std::memcpy(out_challenges, hs + so.chals, static_cast<size_t>(n) * L * 4);
  if (out_finals) std::memcpy(out_finals, hs + so.finals, static_cast<size_t>(1 + S->K) * L * 4);
  if (out_claim0) std::memcpy(out_claim0, hs + so.claim0, L * 4);
  if (out_checksum) std::memcpy(out_checksum, hs + so.checksum, 8);
  return SC_OK;
}

int sc_split_destroy(sc_split* S) {
  if (!S) return SC_OK;
  cudaSetDevice(S->ctx->device);
  cudaStreamSynchronize(S->ctx->stream);
  for (DevBuf* b : {&S->fold_a, &S->fold_b, &S->partials, &S->state, &S->ext, &S->parts, &S->tail, &S->tail_a, &S->tail_b})
    if (b->p) cudaFree(b->p);
  if (S->host) cudaFreeHost(S->host);
  delete S;
  return SC_OK;
}

}  // extern "C"
