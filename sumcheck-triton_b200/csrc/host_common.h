// Host-side pieces shared by the C ABI translation units: error reporting, the opaque
// handle types, scratch buffers, expression and proof-state layout.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/sumcheck_b200.h"
#include "host_field.h"
#include "prover.cuh"
#include "tables.cuh"

using namespace sc;


namespace sc_host {

inline thread_local std::string g_err;

inline int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define SC_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return fail(SC_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

constexpr int kBlock = 256;
constexpr int kMaxDynSmem = 200 * 1024;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// The batched round kernel's launch shape and launch (instantiated once, in batch.cu):
// threads per block, grid (resident blocks on every SM) and dynamic shared memory for
// requests of up to kmax tables. dmax is the largest degree the instance proves: a degree
// class (2, 4, 7) or 6.
int batch_kernel_setup(int L, int K, int dmax, int kmax, int threads_req, int sm_count, int* threads, int* grid,
                       size_t* smem);
int batch_kernel_launch(int L, int K, int dmax, const sc_field* field, unsigned grid, int threads, size_t smem,
                        cudaStream_t stream, const BatchTickArgs& T);

}  // namespace sc_host

using sc_host::DevBuf;

// Launch shape of the batched kernel for one (L, field kind, degree class, tables): the
// plain path's tail launch (capi.cu) looks it up once per context.
struct TailShape {
  int L, kind, dclass, tables, threads;
  size_t smem;
};

struct sc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  DevBuf fold_a, fold_b, partials, state;
  DevBuf tail;                        // the tail launch's BatchRound and ExprDev
  void* tail_host = nullptr;          // pinned staging of the same
  cudaEvent_t tail_copied = nullptr;  // the staging's last copy to the device
  std::vector<TailShape> tail_shapes;
  uint32_t* host_state = nullptr;  // pinned staging of the proof state
  size_t host_state_bytes = 0;
  // per-launch timing of the round kernels (off by default)
  bool timing = false;
  std::vector<cudaEvent_t> events;   // 2 per launch
  int events_used = 0;
  std::vector<float> launch_ms;      // durations of the launches since the last read
};

struct sc_field {
  HostField hf;
  FieldConsts consts;        // host copy
  FieldConsts* dev = nullptr;
  int device = -1;
  bool has_inverses = true;
};

struct sc_expr {
  int num_vars = 0, num_terms = 0, degree = 0;
  std::vector<int64_t> coeffs;
  std::vector<uint32_t> coeff_limbs;  // num_terms x 8 when given
  std::vector<int32_t> lens, offs, flat;
};

namespace sc_host {

inline int ensure(sc_ctx* ctx, DevBuf& b, size_t bytes) {
  if (bytes <= b.bytes) return SC_OK;
  if (b.p) {
    SC_CUDA(cudaStreamSynchronize(ctx->stream));
    SC_CUDA(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
  }
  size_t want = std::max<size_t>(bytes, 256);
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    b.p = nullptr;
    return fail(SC_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", want, cudaGetErrorString(e));
  }
  b.bytes = want;
  return SC_OK;
}

// Events bracketing one launch when timing is on (pool grows as needed).
inline int timing_begin(sc_ctx* ctx, cudaEvent_t* start) {
  if (!ctx->timing) return SC_OK;
  while (static_cast<int>(ctx->events.size()) < ctx->events_used + 2) {
    cudaEvent_t e;
    SC_CUDA(cudaEventCreate(&e));
    ctx->events.push_back(e);
  }
  *start = ctx->events[ctx->events_used++];
  SC_CUDA(cudaEventRecord(*start, ctx->stream));
  return SC_OK;
}

inline int timing_end(sc_ctx* ctx) {
  if (!ctx->timing) return SC_OK;
  SC_CUDA(cudaEventRecord(ctx->events[ctx->events_used++], ctx->stream));
  return SC_OK;
}

// After a synchronisation: turn recorded event pairs into durations.
inline int timing_collect(sc_ctx* ctx) {
  if (!ctx->timing) return SC_OK;
  for (int i = 0; i + 1 < ctx->events_used; i += 2) {
    float ms = 0.f;
    SC_CUDA(cudaEventElapsedTime(&ms, ctx->events[i], ctx->events[i + 1]));
    ctx->launch_ms.push_back(ms);
  }
  ctx->events_used = 0;
  return SC_OK;
}

// ---- compile-time instantiations: limb count L, field kind K, degree class DMAX ----

inline int degree_class(int d) { return d <= 2 ? 2 : (d <= 4 ? 4 : 7); }

inline int field_kind(const uint32_t* p, int L) {
  if (L == 2 && p[0] == 1u && p[1] == 0xFFFFFFFFu) return kFieldGoldilocks;
  if (L == 4 && p[0] == 0xFFFFFFFFu && p[1] == 0xFFFFFFFFu && p[2] == 0xFFFFFFFFu && p[3] == 0x7FFFFFFFu)
    return kFieldMersenne127;
  return kFieldGeneric;
}

// Calls Fn<L, K, DMAX>::run(args...) for the runtime (L, K, DMAX class).
template <template <int, int, int> class Fn, int L, int K, typename... Args>
inline int dispatch_degree(int dclass, Args&&... args) {
  switch (dclass) {
    case 2: return Fn<L, K, 2>::run(args...);
    case 4: return Fn<L, K, 4>::run(args...);
    default: return Fn<L, K, 7>::run(args...);
  }
}

template <template <int, int, int> class Fn, typename... Args>
inline int dispatch(int L, int K, int dclass, Args&&... args) {
  switch (L) {
    case 1: return dispatch_degree<Fn, 1, kFieldGeneric>(dclass, args...);
    case 2:
      return K == kFieldGoldilocks ? dispatch_degree<Fn, 2, kFieldGoldilocks>(dclass, args...)
                                   : dispatch_degree<Fn, 2, kFieldGeneric>(dclass, args...);
    case 4:
      return K == kFieldMersenne127 ? dispatch_degree<Fn, 4, kFieldMersenne127>(dclass, args...)
                                    : dispatch_degree<Fn, 4, kFieldGeneric>(dclass, args...);
    default: return dispatch_degree<Fn, 8, kFieldGeneric>(dclass, args...);
  }
}

// Calls Fn for every instantiation (set-up of kernel attributes).
template <template <int, int, int> class Fn>
inline int for_each_instance() {
  const int combos[6][2] = {{1, kFieldGeneric}, {2, kFieldGeneric}, {2, kFieldGoldilocks},
                            {4, kFieldGeneric}, {4, kFieldMersenne127}, {8, kFieldGeneric}};
  for (const auto& c : combos)
    for (int dc : {2, 4, 7}) {
      const int rc = dispatch<Fn>(c[0], c[1], dc);
      if (rc) return rc;
    }
  return SC_OK;
}

template <int L, int K, int D>
struct SetRoundAttrs {
  static int run() {
    SC_CUDA(cudaFuncSetAttribute(round_kernel<L, K, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem));
    if constexpr (D == 4) {  // the shape kernels (the 2-limb Goldilocks ones stage pairs in shared memory)
      SC_CUDA(cudaFuncSetAttribute(round_kernel<L, K, 4, kShapeZerocheck>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kMaxDynSmem));
      SC_CUDA(cudaFuncSetAttribute(round_kernel<L, K, 4, kShapeAbcg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kMaxDynSmem));
    }
    return SC_OK;
  }
};

// Montgomery image of a small non-negative integer.
inline void mont_small(const HostField& hf, const uint32_t* r2, uint64_t v, uint32_t* out) {
  uint32_t w[2] = {static_cast<uint32_t>(v), static_cast<uint32_t>(v >> 32)};
  uint32_t red[8];
  hf.reduce(w, 2, red);
  hf.mul(red, r2, out);
}

inline void mont_pow(const HostField& hf, const uint32_t* base, const uint32_t* e, const uint32_t* one,
              uint32_t* out) {
  uint32_t acc[8];
  std::memcpy(acc, one, 32);
  for (int w = hf.L - 1; w >= 0; --w)
    for (int b = 31; b >= 0; --b) {
      hf.mul(acc, acc, acc);
      if ((e[w] >> b) & 1u) hf.mul(acc, base, acc);
    }
  std::memcpy(out, acc, 4 * hf.L);
}

// Checks the CIOS exactness bound: (p - 1) 2^32 + p < 2^(32 (L + 1)).
inline bool cios_bound_holds(const HostField& hf) {
  const int L = hf.L;
  uint32_t x[10] = {0};
  uint32_t pm1[8];
  std::memcpy(pm1, hf.p, 4 * L);
  pm1[0] -= 1;  // p odd, so no borrow
  for (int i = 0; i < L; ++i) x[i + 1] = pm1[i];
  uint64_t c = 0;
  for (int i = 0; i < L + 2; ++i) {
    uint64_t s = static_cast<uint64_t>(x[i]) + (i < L ? hf.p[i] : 0u) + c;
    x[i] = static_cast<uint32_t>(s);
    c = s >> 32;
  }
  return x[L + 1] == 0 && c == 0;
}

// Instruction-count estimates of one product and one modular add (for the choices below).
inline int mul_cost(int L, int K) {
  return K == kFieldGoldilocks ? 16 : (K == kFieldMersenne127 ? 60 : (L == 1 ? 10 : 4 * L * L + 8 * L));
}
inline int add_cost(int L) { return 3 * L + 4; }

// Whether a term of length len in an expression of degree d is cheaper evaluated at points
// 0..len and extrapolated by forward differences than evaluated at every point 0..d.
inline bool extrapolate_term(int len, int d, int L, int K) {
  if (len >= d) return false;
  const int m = mul_cost(L, K), a = add_cost(L);
  const int direct = (len - 1) * (d + 1) * m + len * d * a;
  const int extrap = (len - 1) * (len + 1) * m + len * len * a + (len * (len + 1) / 2 + d * len) * a;
  return extrap < direct;
}

// Matches the expression against the compile-time shapes (prover.cuh: Shape). Returns the
// shape (kShapeGeneric when none matches) and fills role[] with the table of every role.
// Coefficients must be exactly +1 (and -1 for the zerocheck's S4 X3 term); every table used
// once per term, every role a different table.
inline int match_shape(const sc_expr& ex, uint8_t* role) {
  if (!ex.coeff_limbs.empty() || ex.degree != 4) return kShapeGeneric;
  const int T = ex.num_terms;
  std::vector<std::vector<int>> terms(T);
  for (int i = 0; i < T; ++i) {
    terms[i].assign(ex.flat.begin() + ex.offs[i], ex.flat.begin() + ex.offs[i] + ex.lens[i]);
    std::vector<int> u = terms[i];
    std::sort(u.begin(), u.end());
    if (std::adjacent_find(u.begin(), u.end()) != u.end()) return kShapeGeneric;  // repeated factor
  }
  auto has = [](const std::vector<int>& v, int x) { return std::find(v.begin(), v.end(), x) != v.end(); };
  // the table common to every term
  int common = -1;
  for (int k = 0; k < ex.num_vars && common < 0; ++k) {
    bool all = true;
    for (int i = 0; i < T && all; ++i) all = has(terms[i], k);
    if (all) common = k;
  }
  if (common < 0) return kShapeGeneric;
  std::vector<std::vector<int>> rest(T);
  for (int i = 0; i < T; ++i)
    for (int x : terms[i])
      if (x != common) rest[i].push_back(x);
  auto distinct_all = [&](const std::vector<int>& r) {
    if (static_cast<int>(r.size()) != ex.num_vars) return false;
    std::vector<int> u = r;
    std::sort(u.begin(), u.end());
    for (int k = 0; k < ex.num_vars; ++k)
      if (u[k] != k) return false;
    return true;
  };
  if (T == 2 && ex.num_vars == 6 && ex.coeffs[0] == 1 && ex.coeffs[1] == 1) {
    const int i3 = rest[0].size() == 3 ? 0 : 1;
    const std::vector<int>& a = rest[i3];
    const std::vector<int>& b = rest[1 - i3];
    if (a.size() != 3 || b.size() != 2) return kShapeGeneric;
    const std::vector<int> r = {a[0], a[1], a[2], common, b[0], b[1]};
    if (!distinct_all(r)) return kShapeGeneric;
    for (int i = 0; i < 6; ++i) role[i] = static_cast<uint8_t>(r[i]);
    return kShapeAbcg;
  }
  if (T == 5 && ex.num_vars == 9) {
    int m = -1, c1 = -1, neg = -1;
    std::vector<int> pos2;
    for (int i = 0; i < T; ++i) {
      const size_t n = rest[i].size();
      const int64_t c = ex.coeffs[i];
      if (n == 3 && c == 1 && m < 0) m = i;
      else if (n == 1 && c == 1 && c1 < 0) c1 = i;
      else if (n == 2 && c == -1 && neg < 0) neg = i;
      else if (n == 2 && c == 1) pos2.push_back(i);
      else return kShapeGeneric;
    }
    if (m < 0 || c1 < 0 || neg < 0 || pos2.size() != 2) return kShapeGeneric;
    const std::vector<int>& M = rest[m];
    int x[2], sel[2];
    for (int j = 0; j < 2; ++j) {
      const std::vector<int>& P = rest[pos2[j]];
      const bool in0 = has(M, P[0]), in1 = has(M, P[1]);
      if (in0 == in1) return kShapeGeneric;  // exactly one factor shared with the degree-3 term
      x[j] = in0 ? P[0] : P[1];
      sel[j] = in0 ? P[1] : P[0];
    }
    if (x[0] == x[1]) return kShapeGeneric;
    int mr = -1;
    for (int v : M)
      if (v != x[0] && v != x[1]) mr = v;
    const std::vector<int> r = {sel[0], x[0], common, sel[1], x[1], mr, rest[neg][0], rest[neg][1], rest[c1][0]};
    if (mr < 0 || !distinct_all(r)) return kShapeGeneric;
    for (int i = 0; i < 9; ++i) role[i] = static_cast<uint8_t>(r[i]);
    return kShapeZerocheck;
  }
  return kShapeGeneric;
}

template <int L>
inline void build_expr_dev(const sc_expr& ex, const sc_field& f, ExprDev& E) {
  std::memset(&E, 0, sizeof(E));
  E.shape = match_shape(ex, E.role);
  E.num_vars = ex.num_vars;
  E.num_terms = ex.num_terms;
  E.degree = ex.degree;
  const HostField& hf = f.hf;
  const int K = field_kind(hf.p, L);
  for (int i = 0; i < ex.num_terms; ++i) E.term_extrap[i] = extrapolate_term(ex.lens[i], ex.degree, L, K) ? 1 : 0;
  const int mul_cost = ::sc_host::mul_cost(L, K), add_cost = ::sc_host::add_cost(L);
  for (int i = 0; i < ex.num_terms; ++i) {
    E.term_len[i] = static_cast<uint8_t>(ex.lens[i]);
    E.term_off[i] = static_cast<uint8_t>(ex.offs[i]);
    bool use_mont = !ex.coeff_limbs.empty();
    const int64_t c = ex.coeffs[i];
    if (!use_mont) {
      if (c == 1) {
        E.coeff_kind[i] = kCoeffPlus;
      } else if (c == -1) {
        E.coeff_kind[i] = kCoeffMinus;
      } else if (c > -(int64_t{1} << 31) && c < (int64_t{1} << 31)) {
        const uint64_t m = c < 0 ? static_cast<uint64_t>(-c) : static_cast<uint64_t>(c);
        const int bits = m ? 64 - __builtin_clzll(m) : 0;
        const int chain = (bits > 0 ? bits - 1 : 0) + (m ? __builtin_popcountll(m) - 1 : 0) + (c < 0);
        if (chain * add_cost <= mul_cost) {
          E.coeff_kind[i] = kCoeffSmall;
          E.coeff_small[i] = static_cast<int32_t>(c);
        } else {
          use_mont = true;
        }
      } else {
        use_mont = true;
      }
    }
    if (use_mont) {
      E.coeff_kind[i] = kCoeffMont;
      uint32_t red[8];
      if (!ex.coeff_limbs.empty()) {
        hf.reduce(&ex.coeff_limbs[8 * i], 8, red);
      } else {
        const uint64_t m = c < 0 ? static_cast<uint64_t>(-(c + 1)) + 1u : static_cast<uint64_t>(c);
        uint32_t w[2] = {static_cast<uint32_t>(m), static_cast<uint32_t>(m >> 32)};
        hf.reduce(w, 2, red);
        if (c < 0) hf.neg(red, red);
      }
      uint32_t mont[8];
      hf.mul(red, f.consts.r2, mont);
      for (int l = 0; l < L; ++l) E.coeff_mont[i][l] = mont[l];
    }
  }
  for (size_t i = 0; i < ex.flat.size(); ++i) E.flat[i] = static_cast<uint8_t>(ex.flat[i]);
}

struct StateOffsets {
  size_t counter, status, checksum, polys, chals, finals, claim0, claim, total_words;
};

inline StateOffsets state_offsets(int n, int K, int L) {
  StateOffsets o;
  o.counter = 0;
  o.status = 1;
  o.checksum = 2;  // u64 at word 2 (8-byte aligned)
  o.polys = 4;
  o.chals = o.polys + static_cast<size_t>(n) * kMaxPoints * L;
  o.finals = o.chals + static_cast<size_t>(n) * L;
  o.claim0 = o.finals + static_cast<size_t>(1 + K) * L;
  o.claim = o.claim0 + L;
  o.total_words = o.claim + L;
  return o;
}


// ---- transcripts: a proof stopped at a round boundary, resumable from the same tables
//
// A transcript is the header below followed by the proof-state words (state_offsets
// layout) as the round kernels leave them after round rounds_done - 1: checksum so far,
// g_j for j < rounds_done, r_j for j < rounds_done, claim0, and the claim the next round
// meets. That is all a later call needs: the challenges refold the tables to the round it
// continues from, and finalize_round goes on adding to the same checksum.
constexpr uint32_t kTranscriptMagic = 0x31524353u;  // "SCR1"
constexpr int kTranscriptHeader = 16;
enum TranscriptWord {
  kTwMagic = 0, kTwHeaderWords = 1, kTwLimbs = 2, kTwRounds = 3, kTwVars = 4, kTwDegree = 5, kTwMode = 6,
  kTwDone = 7, kTwExprDigest = 8, kTwFieldDigest = 10, kTwTablesTag = 12, kTwStateWords = 14,
};

constexpr uint64_t kFnvBasis = 0xcbf29ce484222325ull;

inline uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
  return h;
}

template <typename T>
inline uint64_t fnv1a_vec(uint64_t h, const std::vector<T>& v) {
  const uint64_t n = v.size();
  h = fnv1a(h, &n, sizeof(n));
  return v.empty() ? h : fnv1a(h, v.data(), v.size() * sizeof(T));
}

inline uint64_t expr_digest(const sc_expr& e) {
  const int32_t dims[3] = {e.num_vars, e.num_terms, e.degree};
  uint64_t h = fnv1a(kFnvBasis, dims, sizeof(dims));
  h = fnv1a_vec(h, e.coeffs);
  h = fnv1a_vec(h, e.coeff_limbs);
  h = fnv1a_vec(h, e.lens);
  h = fnv1a_vec(h, e.offs);
  return fnv1a_vec(h, e.flat);
}

inline uint64_t field_digest(const HostField& hf) {
  const int32_t L = hf.L;
  uint64_t h = fnv1a(kFnvBasis, &L, sizeof(L));
  return fnv1a(h, hf.p, static_cast<size_t>(L) * 4);
}

// The tag of seeded tables (sc_tables_tag; the server's requests carry it).
inline uint64_t seeded_tables_tag(int num_tables, const int32_t* kinds, uint64_t seed) {
  const char dom[] = "sc:seeded-tables:v1";
  uint64_t h = fnv1a(kFnvBasis, dom, sizeof(dom) - 1);
  const int32_t k = num_tables;
  h = fnv1a(h, &k, sizeof(k));
  h = fnv1a(h, kinds, static_cast<size_t>(num_tables) * 4);
  return fnv1a(h, &seed, sizeof(seed));
}

inline size_t transcript_words(int n, int K, int L) {
  return kTranscriptHeader + state_offsets(n, K, L).total_words;
}

inline void tw_put64(uint32_t* t, int w, uint64_t v) {
  t[w] = static_cast<uint32_t>(v);
  t[w + 1] = static_cast<uint32_t>(v >> 32);
}
inline uint64_t tw_get64(const uint32_t* t, int w) { return t[w] | (static_cast<uint64_t>(t[w + 1]) << 32); }

inline void transcript_header(uint32_t* t, const HostField& hf, const sc_expr& ex, int n, int mode, int done,
                              uint64_t tag) {
  std::memset(t, 0, kTranscriptHeader * 4);
  t[kTwMagic] = kTranscriptMagic;
  t[kTwHeaderWords] = kTranscriptHeader;
  t[kTwLimbs] = static_cast<uint32_t>(hf.L);
  t[kTwRounds] = static_cast<uint32_t>(n);
  t[kTwVars] = static_cast<uint32_t>(ex.num_vars);
  t[kTwDegree] = static_cast<uint32_t>(ex.degree);
  t[kTwMode] = static_cast<uint32_t>(mode);
  t[kTwDone] = static_cast<uint32_t>(done);
  tw_put64(t, kTwExprDigest, expr_digest(ex));
  tw_put64(t, kTwFieldDigest, field_digest(hf));
  tw_put64(t, kTwTablesTag, tag);
  t[kTwStateWords] = static_cast<uint32_t>(state_offsets(n, ex.num_vars, hf.L).total_words);
}

// A transcript's header, parsed and checked for self-consistency (not against a proof).
struct TranscriptInfo {
  int L = 0, n = 0, K = 0, d = 0, mode = 0, done = 0;
  uint64_t expr_digest = 0, field_digest = 0, tag = 0;
};

inline int transcript_parse(const uint32_t* t, uint64_t words, TranscriptInfo* out) {
  if (!t) return fail(SC_ERR_INVALID, "NULL transcript");
  if (words < static_cast<uint64_t>(kTranscriptHeader) || t[kTwMagic] != kTranscriptMagic ||
      t[kTwHeaderWords] != static_cast<uint32_t>(kTranscriptHeader))
    return fail(SC_ERR_INVALID, "not a transcript (bad magic or header)");
  TranscriptInfo I;
  I.L = static_cast<int>(t[kTwLimbs]);
  I.n = static_cast<int>(t[kTwRounds]);
  I.K = static_cast<int>(t[kTwVars]);
  I.d = static_cast<int>(t[kTwDegree]);
  I.mode = static_cast<int>(t[kTwMode]);
  I.done = static_cast<int>(t[kTwDone]);
  if (!(I.L == 1 || I.L == 2 || I.L == 4 || I.L == 8) || I.n < 1 || I.n > kMaxRounds || I.K < 1 || I.K > kMaxVars ||
      I.d < 1 || I.d > kMaxPoints - 1 || I.mode < SC_CHALLENGE_SHA3 || I.mode > SC_CHALLENGE_EXPLICIT || I.done < 0 ||
      I.done > I.n)
    return fail(SC_ERR_INVALID, "transcript header out of range");
  if (t[kTwStateWords] != state_offsets(I.n, I.K, I.L).total_words || words < transcript_words(I.n, I.K, I.L))
    return fail(SC_ERR_INVALID, "transcript of %llu words is shorter than its header says",
                static_cast<unsigned long long>(words));
  I.expr_digest = tw_get64(t, kTwExprDigest);
  I.field_digest = tw_get64(t, kTwFieldDigest);
  I.tag = tw_get64(t, kTwTablesTag);
  *out = I;
  return SC_OK;
}

// The transcript belongs to this field and expression.
inline int transcript_match(const TranscriptInfo& I, const HostField& hf, const sc_expr& ex) {
  if (I.L != hf.L || I.field_digest != field_digest(hf)) return fail(SC_ERR_INVALID, "transcript is of another field");
  if (I.K != ex.num_vars || I.d != ex.degree || I.expr_digest != expr_digest(ex))
    return fail(SC_ERR_INVALID, "transcript is of another expression");
  return SC_OK;
}

// Proves rounds [first, stop) of a proof on the context's stream. state_io (host,
// state_offsets words) is uploaded before -- the state after round first - 1, zeros for
// first = 0 -- and downloaded after. T_0 is first folded up to T_{first-1} with the
// recorded challenges. Defined in capi.cu.
int prove_segment(sc_ctx* ctx, const sc_field* field, const sc_expr* expr, int n, const uint32_t* tables, int mode,
                  const uint32_t* explicit_ch, int first, int stop, uint32_t* state_io);

// Folds T_0 (tables) to T_{j-1} on `stream` with r_0..r_{j-2} from chals_dev (L words each):
// T_i goes to fold_a for odd i and fold_b for even i, where round j's kernel reads it.
// Nothing to do for j <= 1. Defined in capi.cu.
int resume_folds(const sc_field* field, int n, int num_tables, const uint32_t* tables, uint32_t* fold_a,
                 uint32_t* fold_b, const uint32_t* chals_dev, int j, int sm_count, cudaStream_t stream);

}  // namespace sc_host
