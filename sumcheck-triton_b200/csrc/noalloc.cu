// sc_prove_noalloc: one proof with no device (or pinned host) allocation at all.
//
// Who needs it: callers that cannot call cudaMalloc -- code running inside another
// framework's memory pool or under a strict device-memory budget, plug-ins that may not
// grow the process's device footprint after start-up, or hosts that forbid allocation on
// the proving path. sc_prove grows its context's scratch with cudaMalloc and stages the
// results in pinned host memory; this variant does neither.
//
// Its scratch -- the field constants, the proof state, the block partials and the two fold
// buffers -- lives in one file-scope __device__ array of kNoAllocScratchBytes (32 MiB).
// Every GPU that loads the library holds that array until the process exits. A proof fits
// when K L 2^n (3/4) words of fold buffers plus the small rest fit; larger proofs are
// rejected with SC_ERR_UNSUPPORTED before anything runs.
//
// In host code the array's name stands in for the device object, it is not a device
// address: the first call on each device (with that device current) asks the runtime for
// the address with cudaGetSymbolAddress and caches it, and sets the round kernels'
// attributes. Make that first call before any stream capture. The cached address belongs
// to the device's primary context: do not reset that context (cudaDeviceReset) after the
// first call on the device, or later calls would launch into an unmapped address.
// The call is synchronous: it returns once the results are in the caller's arrays.
// All calls share the one array and it keeps the last call's contents; what must start at
// zero (the proof state's counter, status and checksum) is cleared by every call. Two
// calls whose work overlaps on the same GPU race on the array: issue them on one stream,
// or wait for one before starting the next.
#include <mutex>

#include "host_common.h"

using namespace sc;
using namespace sc_host;

namespace {
constexpr size_t kNoAllocScratchBytes = size_t{32} << 20;
constexpr int kNoAllocMaxBlocks = 1184;  // 148 SMs x 8
constexpr int kMaxDevices = 64;
}  // namespace

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocScratchBytes / 4];

namespace {

std::mutex g_noalloc_mu;
uint32_t* g_noalloc_ptr[kMaxDevices] = {};


// Device address of the scratch array on `device` (the device must be current).
int noalloc_scratch(int device, uint32_t** out) {
  if (device < 0 || device >= kMaxDevices) return fail(SC_ERR_INVALID, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(SC_ERR_CUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", device, cudaGetErrorString(e));
    const int rc = for_each_instance<SetRoundAttrs>();
    if (rc) return rc;
    g_noalloc_ptr[device] = static_cast<uint32_t*>(p);
  }
  *out = g_noalloc_ptr[device];
  return SC_OK;
}

constexpr size_t align64(size_t w) { return (w + 63) & ~size_t{63}; }  // 256-byte steps

constexpr uint64_t kNoAllocSkip1MinPairs = uint64_t{1} << 12;

template <int L, int K, int DMAX>
struct NoallocRun {
static int run(sc_ctx* ctx, const sc_field* f, const sc_expr* ex, int n, const uint32_t* tables, int mode,
               const uint32_t* explicit_ch, uint32_t* out_polys, uint32_t* out_ch, uint32_t* out_finals,
               uint32_t* out_claim0, uint64_t* out_checksum) {
  const int K_ = ex->num_vars, d = ex->degree;
  const uint64_t N = uint64_t{1} << n;
  uint32_t* base = nullptr;
  int rc;
  if ((rc = noalloc_scratch(ctx->device, &base))) return rc;  // first call on a device: set-up
  int threads = kernel_threads(L);
  const int per_thread = round_smem_words_per_thread(K_, L) * 4;
  while (threads > 32 && threads * per_thread > kMaxDynSmem) threads -= 32;
  const size_t smem = static_cast<size_t>(threads) * per_thread;
  int bps = 0;
  SC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, round_kernel<L, K, DMAX>, threads, smem));
  if (bps < 1) return fail(SC_ERR_UNSUPPORTED, "round kernel does not fit on an SM (K=%d, L=%d)", K_, L);
  const uint64_t grid_max = std::min<uint64_t>(static_cast<uint64_t>(bps) * ctx->sm_count, kNoAllocMaxBlocks);

  // carve the scratch array: field constants, proof state, partials, fold A, fold B
  const StateOffsets so = state_offsets(n, K_, L);
  const size_t w_fc = 0;
  const size_t w_state = w_fc + align64(sizeof(FieldConsts) / 4);
  const size_t w_part = w_state + align64(so.total_words);
  const size_t w_a = w_part + align64(grid_max * kMaxPoints * L);
  const size_t w_b = w_a + align64(n >= 2 ? static_cast<size_t>(K_) * L * (N / 2) : 0);
  const size_t w_end = w_b + align64(n >= 3 ? static_cast<size_t>(K_) * L * (N / 4) : 0);
  if (w_end * 4 > kNoAllocScratchBytes)
    return fail(SC_ERR_UNSUPPORTED,
                "sc_prove_noalloc: this proof (%d tables, %d limbs, 2^%d entries) needs %zu bytes of scratch; "
                "the no-allocation scratch holds %zu bytes (use sc_prove)",
                K_, L, n, w_end * 4, kNoAllocScratchBytes);
  ExprDev E;
  build_expr_dev<L>(*ex, *f, E);
  FieldParams<L, K> F;
  for (int l = 0; l < L; ++l) F.p[l] = f->hf.p[l];
  F.np = f->hf.np;

  uint32_t* st = base + w_state;
  SC_CUDA(cudaMemcpyAsync(base + w_fc, &f->consts, sizeof(FieldConsts), cudaMemcpyHostToDevice, ctx->stream));
  SC_CUDA(cudaMemsetAsync(st, 0, so.total_words * 4, ctx->stream));
  if (mode == SC_CHALLENGE_EXPLICIT)
    SC_CUDA(cudaMemcpyAsync(st + so.chals, explicit_ch, static_cast<size_t>(n) * L * 4, cudaMemcpyHostToDevice,
                            ctx->stream));

  RoundArgs A;
  std::memset(&A, 0, sizeof(A));
  A.num_rounds = n;
  A.mode = mode;
  A.partials = base + w_part;
  A.fc = reinterpret_cast<const FieldConsts*>(base + w_fc);
  A.st.counter = st + so.counter;
  A.st.status = st + so.status;
  A.st.checksum = reinterpret_cast<uint64_t*>(st + so.checksum);
  A.st.polys = st + so.polys;
  A.st.chals = st + so.chals;
  A.st.finals = st + so.finals;
  A.st.claim0 = st + so.claim0;
  A.st.claim = st + so.claim;
  const uint32_t* prev = tables;
  for (int j = 0; j < n; ++j) {
    A.round = j;
    A.pairs = N >> (j + 1);
    A.skip1 = (j >= 1 && (N >> (j + 1)) >= kNoAllocSkip1MinPairs) ? 1 : 0;
    A.want_claim = (j + 1 < n && (N >> (j + 2)) >= kNoAllocSkip1MinPairs) ? 1 : 0;
    if (j == 0) {
      A.fold = 0;
      A.src = tables;
      A.dst = nullptr;
      A.src_len = N;
    } else {
      A.fold = 1;
      A.src = prev;
      A.src_len = N >> (j - 1);
      A.dst = base + ((j & 1) ? w_a : w_b);
      prev = A.dst;
    }
    const uint64_t want = (A.pairs + threads - 1) / threads;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(want, grid_max));
    round_kernel<L, K, DMAX><<<grid, threads, smem, ctx->stream>>>(A, E, F);
    SC_CUDA(cudaGetLastError());
  }
  // results straight into the caller's arrays (no staging buffer)
  uint32_t status = 0;
  SC_CUDA(cudaMemcpyAsync(&status, st + so.status, 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (out_polys)
    SC_CUDA(cudaMemcpy2DAsync(out_polys, static_cast<size_t>(d + 1) * L * 4, st + so.polys,
                              static_cast<size_t>(kMaxPoints) * L * 4, static_cast<size_t>(d + 1) * L * 4, n,
                              cudaMemcpyDeviceToHost, ctx->stream));
  if (out_ch)
    SC_CUDA(cudaMemcpyAsync(out_ch, st + so.chals, static_cast<size_t>(n) * L * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (out_finals)
    SC_CUDA(cudaMemcpyAsync(out_finals, st + so.finals, static_cast<size_t>(1 + K_) * L * 4, cudaMemcpyDeviceToHost,
                            ctx->stream));
  if (out_claim0) SC_CUDA(cudaMemcpyAsync(out_claim0, st + so.claim0, L * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (out_checksum) SC_CUDA(cudaMemcpyAsync(out_checksum, st + so.checksum, 8, cudaMemcpyDeviceToHost, ctx->stream));
  SC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (status) return fail(SC_ERR_DEVICE, "device status %u", status);
  return SC_OK;
}
};

}  // namespace

extern "C" int sc_prove_noalloc(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int num_rounds,
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
  SC_CUDA(cudaSetDevice(ctx->device));
  return dispatch<NoallocRun>(field->hf.L, field_kind(field->hf.p, field->hf.L), degree_class(expr->degree), ctx,
                              field, expr, num_rounds, tables_dev, challenge_mode, explicit_challenges,
                              out_round_polys, out_challenges, out_finals, out_claim0, out_checksum);
}
