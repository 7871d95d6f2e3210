// The SumCheck round kernel and its finalisation.
//
// One launch per round j does the whole round, with no host round trip:
//
//   1. fold (j >= 1): each thread reads 4 consecutive entries of every table of round j-1
//      (one 128-bit load per limb plane), folds them with r_{j-1} into the pair
//      (T_j[2i], T_j[2i+1]) and writes that pair back (the fold of the previous round,
//      reference field_sumcheck.cu:677-694, fused into this round's read);
//   2. evaluate: extends every table's pair to t = 0..d (v(t) = v(t-1) + (o - e); reference
//      field_sumcheck.cu:326-348) and evaluates the constraint at each point
//      (field_sumcheck.cu:389-590), accumulating d+1 sums per thread (see eval_pair for the
//      exact-arithmetic shortcuts: extrapolated low-degree terms, g(1) from the claim);
//   3. reduce: warp shuffles, then shared memory, then one partial per block in global
//      memory; the last block to finish (atomic ticket) sums the partials -- a single-pass
//      grid reduction in place of the reference's log-depth launch tree
//      (field_sumcheck.cu:635-675, :996-1010);
//   4. finalise (last block only): stores g_j(0..d), adds the round's checksum, derives r_j
//      by SHA3 over the round polynomial on the device (field_sumcheck.cu:857-907), and when
//      needed g_j(r_j) (the next round's claim) and, in the last round, the final claim and
//      the folded values f_k(r).
//
// Tables are limb-planar: table k, limb l is the u32 plane at (k * L + l) * len.
// Kernels are templates over the limb count L, the field kind K (a special reduction for
// Goldilocks) and DMAX, the largest degree the launch handles (register arrays of DMAX + 1
// points; the host picks the smallest class >= the expression's degree).
#pragma once
#include <cstdint>
#include <type_traits>

#include "field.cuh"
#include "keccak.cuh"

namespace sc {

constexpr int kMaxVars = 32;
constexpr int kMaxTerms = 32;
constexpr int kMaxFlat = 128;
constexpr int kMaxRounds = 40;

enum ChallengeMode : int32_t { kChallengeSha3 = 0, kChallengeFixed = 1, kChallengeExplicit = 2 };

// Coefficient handling per term: +1 / -1 are an add / a subtract; other small values an
// addition chain; anything else a product with the coefficient's Montgomery image. The
// scaling is applied once per pair to the first factor (value and difference), not per point.
enum CoeffKind : uint8_t { kCoeffPlus = 0, kCoeffMinus = 1, kCoeffSmall = 2, kCoeffMont = 3 };

// Constants of one field that only the finalisation needs (device memory, per field).
struct FieldConsts {
  uint32_t p[kMaxLimbs];
  uint32_t np;
  uint32_t limbs;
  uint32_t p_small;                          // p if p < 2^32, else 0
  uint32_t one[kMaxLimbs];                   // R mod p
  uint32_t r2[kMaxLimbs];                    // R^2 mod p
  uint32_t pts[kMaxPoints][kMaxLimbs];       // Montgomery image of t = 0..7
  uint32_t kdig[8][kMaxLimbs];               // R^2 2^(32 i) mod p: digest word i
  uint32_t lag[kMaxPoints][kMaxPoints][kMaxLimbs];  // lag[d][t] = 1 / prod_{s<=d, s!=t} (t - s)
};

// A compiled expression for one field (kernel parameter: lives in the constant bank).
struct ExprDev {
  int32_t num_vars;
  int32_t num_terms;
  int32_t degree;
  int32_t pad;
  uint8_t term_len[kMaxTerms];
  uint8_t term_off[kMaxTerms];
  uint8_t flat[kMaxFlat];
  uint8_t coeff_kind[kMaxTerms];
  uint8_t term_extrap[kMaxTerms];   // 1: evaluate points 0..len only, extrapolate the rest
  int32_t coeff_small[kMaxTerms];
  uint32_t coeff_mont[kMaxTerms][kMaxLimbs];
  int32_t shape;                    // Shape the host matched (kShapeGeneric: none)
  uint8_t role[16];                 // shape kernels: table index of each role
};

// Expression shapes with a compile-time evaluator (the host matches the term structure and
// maps tables to roles; any table order and any order of the symmetric factors matches):
//   kShapeZerocheck  F (X1 S1 + X2 S2 + X1 X2 M - X3 S4 + S5)   roles S1 X1 F S2 X2 M S4 X3 S5
//                    evaluated as F (X1 (S1 + M X2) + S2 X2 - S4 X3 + S5): 5 products a point
//                    (the vanilla zerocheck gate, src/zkduel/workloads.py:37-43)
//   kShapeAbcg       G (A B C + D E)                              roles A B C G D E
//                    4 products a point (poly_abcg_plus_deg, workloads.py:32)
enum Shape : int32_t { kShapeGeneric = 0, kShapeZerocheck = 1, kShapeAbcg = 2 };

__host__ __device__ constexpr int shape_tables(int shape) {
  return shape == kShapeZerocheck ? 9 : (shape == kShapeAbcg ? 6 : 0);
}

// Device-detected errors, or-ed into ProofState::status (the host fails the call with
// SC_ERR_DEVICE when it reads a nonzero status):
//   kStatusClaim  a round that evaluated g(1) directly and was given a claim to meet
//                 (RoundArgs::check_claim) found g_j(0) + g_j(1) != the claim -- the tables
//                 are not the ones the recorded rounds were proved on, or the recorded claim
//                 was altered (a resumed transcript's first round checks this).
constexpr uint32_t kStatusClaim = 1u;

// Per-proof device state, all Montgomery limbs (written by the finalisation).
struct ProofState {
  uint32_t* counter;     // block tickets of the running round, reset to 0 after each round
  uint64_t* checksum;    // sum over rounds and points of (i + 1) limb_i
  uint32_t* polys;       // [n][kMaxPoints][L]
  uint32_t* chals;       // [n][L]
  uint32_t* finals;      // [1 + K][L]: g_{n-1}(r_{n-1}), then f_k(r) for every table
  uint32_t* claim0;      // [L]
  uint32_t* status;      // nonzero on a device-detected error: kStatusClaim
  uint32_t* claim;       // [L]: g_{j-1}(r_{j-1}), the claim round j's g(0) + g(1) must meet
};

struct RoundArgs {
  const uint32_t* src;   // T_{j-1} when folding, else T_j
  uint32_t* dst;         // T_j when folding, else unused
  uint64_t src_len;      // entries per plane of src
  uint64_t pairs;        // N_j / 2
  int32_t round;
  int32_t num_rounds;
  int32_t fold;
  int32_t mode;          // ChallengeMode
  int32_t skip1;         // g(1) = claim - g(0) instead of evaluating point 1
  int32_t want_claim;    // store g_j(r_j) for the next round
  uint32_t* partials;    // [gridDim.x][kMaxPoints][L]
  const FieldConsts* fc;
  ProofState st;
  uint32_t* ext_out;     // non-null: the round's sums g_j(0..d) go here and the round is not
                         // finalised (one rank of a split proof; the commit finalises it)
  int32_t check_claim;   // with skip1 == 0: check g_j(0) + g_j(1) against st.claim (kStatusClaim)
  int32_t pad;
};

template <int L>
__device__ __forceinline__ Fe<L> ld_fe(const uint32_t* p) {
  Fe<L> r;
#pragma unroll
  for (int i = 0; i < L; ++i) r.w[i] = p[i];
  return r;
}

template <int L>
__device__ __forceinline__ Fe<L> ld_fe_cg(const uint32_t* p) {
  Fe<L> r;
#pragma unroll
  for (int i = 0; i < L; ++i) r.w[i] = __ldcg(p + i);
  return r;
}

template <int L>
__device__ __forceinline__ void st_fe(uint32_t* p, const Fe<L>& a) {
#pragma unroll
  for (int i = 0; i < L; ++i) p[i] = a.w[i];
}

// Shared-memory element of thread `tid` in a [slot][limb][thread] array (conflict-free).
template <int L>
__device__ __forceinline__ Fe<L> sm_get(const uint32_t* sm, int slot, int tid, int nthr) {
  Fe<L> r;
#pragma unroll
  for (int l = 0; l < L; ++l) r.w[l] = sm[(slot * L + l) * nthr + tid];
  return r;
}

template <int L>
__device__ __forceinline__ void sm_put(uint32_t* sm, int slot, int tid, int nthr, const Fe<L>& a) {
#pragma unroll
  for (int l = 0; l < L; ++l) sm[(slot * L + l) * nthr + tid] = a.w[l];
}

template <int L, int K>
__device__ __forceinline__ Fe<L> add_or_sub(const Fe<L>& acc, const Fe<L>& x, bool neg, const FieldParams<L, K>& F) {
  return neg ? fe_sub(acc, x, F) : fe_add(acc, x, F);
}

// The generic evaluator over Goldilocks in lazy arithmetic (field.cuh gl_*): stepped values,
// products and point sums are any representatives in [0, 2^64); the values and differences it
// reads are canonical, and process_pairs makes the point sums canonical after the thread's
// last pair. Measured on B200, the mixed stream's 64-bit group alone: 5.93 against 6.07 ms.
#ifndef SC_GOLD_LAZY_GENERIC
#define SC_GOLD_LAZY_GENERIC 1
#endif
template <int L, int K>
__host__ __device__ constexpr bool lazy_generic() {
  return L == 2 && K == kFieldGoldilocks && SC_GOLD_LAZY_GENERIC;
}
template <bool LZ, int L, int K>
__device__ __forceinline__ Fe<L> lz_add(const Fe<L>& a, const Fe<L>& b, const FieldParams<L, K>& F) {
  if constexpr (LZ) return gl_add(a, b, gold_k(F));
  else return fe_add(a, b, F);
}
template <bool LZ, int L, int K>  // b canonical
__device__ __forceinline__ Fe<L> lz_add_c(const Fe<L>& a, const Fe<L>& b, const FieldParams<L, K>& F) {
  if constexpr (LZ) return gl_add_c(a, b, gold_k(F));
  else return fe_add(a, b, F);
}
template <bool LZ, int L, int K>
__device__ __forceinline__ Fe<L> lz_sub(const Fe<L>& a, const Fe<L>& b, const FieldParams<L, K>& F) {
  if constexpr (LZ) return gl_sub(a, b, gold_k(F));
  else return fe_sub(a, b, F);
}
template <bool LZ, int L, int K>
__device__ __forceinline__ Fe<L> lz_mul(const Fe<L>& a, const Fe<L>& b, const FieldParams<L, K>& F) {
  if constexpr (LZ) return gl_mul(a, b, gold_k(F));
  else return fe_mul(a, b, F);
}
template <bool LZ, int L, int K>
__device__ __forceinline__ Fe<L> lz_add_or_sub(const Fe<L>& acc, const Fe<L>& x, bool neg, const FieldParams<L, K>& F) {
  return neg ? lz_sub<LZ>(acc, x, F) : lz_add<LZ>(acc, x, F);
}

// One pair: acc[t] += expression at point t, for t = 0..d (t = 1 skipped when skip1).
// The values and differences of every table are in shared memory (this thread's slots).
//
// A term of len factors is a polynomial of degree len in t. Evaluated at points 0..last
// (last = d, or len when the host marked the term for extrapolation), each point costs len-1
// products: the factors' values are stepped point to point by one addition of the
// difference. An extrapolated term's points len+1..d come from its forward differences
// (len(len+1)/2 subtractions, then len additions per step) -- exact, since the term is a
// polynomial of degree len; the host marks a term only where that is cheaper than the
// products it replaces. With skip1, point 1 of a directly evaluated term is never formed.
template <int L, int K, int DMAX>
__device__ __forceinline__ void eval_pair(const ExprDev& E, const uint32_t* sv, const uint32_t* sd, int tid, int nthr,
                                          bool skip1, Fe<L> (&acc)[DMAX + 1], const FieldParams<L, K>& F) {
  constexpr bool LZ = lazy_generic<L, K>();
  const int d = E.degree;
  for (int i = 0; i < E.num_terms; ++i) {
    const int off = E.term_off[i];
    const int len = E.term_len[i];
    const int kind = E.coeff_kind[i];
    const bool extrap = E.term_extrap[i] != 0;
    const int last = extrap ? len : d;
    const bool skip_t1 = skip1 && !extrap;
    const bool neg = kind == kCoeffMinus || (kind == kCoeffSmall && E.coeff_small[i] < 0);
    Fe<L> prod[DMAX + 1];
    {
      const int k0 = E.flat[off];
      Fe<L> v = sm_get<L>(sv, k0, tid, nthr);
      Fe<L> df = sm_get<L>(sd, k0, tid, nthr);
      if (kind == kCoeffSmall) {
        const int32_t c = E.coeff_small[i];
        const uint32_t m = c < 0 ? static_cast<uint32_t>(-static_cast<int64_t>(c)) : static_cast<uint32_t>(c);
        v = fe_mul_small(v, m, F);
        df = fe_mul_small(df, m, F);
      } else if (kind == kCoeffMont) {
        Fe<L> cm;
#pragma unroll
        for (int l = 0; l < L; ++l) cm.w[l] = E.coeff_mont[i][l];
        v = fe_mul(v, cm, F);
        df = fe_mul(df, cm, F);
      }
#pragma unroll
      for (int t = 0; t <= DMAX; ++t) {
        if (t > last) break;
        prod[t] = v;
        if (t < last) v = lz_add_c<LZ>(v, df, F);
      }
    }
    for (int f = 1; f < len; ++f) {
      const int k = E.flat[off + f];
      Fe<L> v = sm_get<L>(sv, k, tid, nthr);
      const Fe<L> df = sm_get<L>(sd, k, tid, nthr);
#pragma unroll
      for (int t = 0; t <= DMAX; ++t) {
        if (t > last) break;
        if (!(skip_t1 && t == 1)) prod[t] = lz_mul<LZ>(prod[t], v, F);
        if (t < last) v = lz_add_c<LZ>(v, df, F);
      }
    }
#pragma unroll
    for (int t = 0; t <= DMAX; ++t) {
      if (t > last) break;
      if (skip1 && t == 1) continue;
      acc[t] = lz_add_or_sub<LZ>(acc[t], prod[t], neg, F);
    }
    if (extrap && len < d) {
      // forward differences at 0, in place: prod[m] = Delta^m p(0)
#pragma unroll
      for (int m = 1; m <= DMAX; ++m) {
        if (m > len) break;
#pragma unroll
        for (int t = DMAX; t >= 1; --t) {
          if (t > len || t < m) continue;
          prod[t] = lz_sub<LZ>(prod[t], prod[t - 1], F);
        }
      }
      // step forward: after s steps prod[0] = p(s)
#pragma unroll
      for (int s = 1; s <= DMAX; ++s) {
        if (s > d) break;
#pragma unroll
        for (int m = 0; m < DMAX; ++m) {
          if (m >= len) break;
          prod[m] = lz_add<LZ>(prod[m], prod[m + 1], F);
        }
        if (s > len && !(skip1 && s == 1)) acc[s] = lz_add_or_sub<LZ>(acc[s], prod[0], neg, F);
      }
    }
  }
}

template <int L, int K>
__device__ __forceinline__ Fe<L> shape_value(const Fe<L> (&v)[9], const FieldParams<L, K>& F,
                                             std::integral_constant<int, kShapeZerocheck>) {
  const Fe<L> u = fe_add(v[0], fe_mul(v[5], v[4], F), F);  // S1 + M X2
  Fe<L> s = fe_mul(v[1], u, F);                            // X1 (S1 + M X2)
  s = fe_add(s, fe_mul(v[3], v[4], F), F);                 // + S2 X2
  s = fe_sub(s, fe_mul(v[6], v[7], F), F);                 // - S4 X3
  s = fe_add(s, v[8], F);                                  // + S5
  return fe_mul(v[2], s, F);                               // F (...)
}

template <int L, int K>
__device__ __forceinline__ Fe<L> shape_value(const Fe<L> (&v)[6], const FieldParams<L, K>& F,
                                             std::integral_constant<int, kShapeAbcg>) {
  const Fe<L> s = fe_add(fe_mul(fe_mul(v[0], v[1], F), v[2], F), fe_mul(v[4], v[5], F), F);
  return fe_mul(v[3], s, F);
}

// The same formulas in lazy Goldilocks arithmetic: operands and result in [0, 2^64).
__device__ __forceinline__ Fe<2> shape_value_lazy(const Fe<2> (&v)[9], const GoldK k,
                                                  std::integral_constant<int, kShapeZerocheck>) {
  const Fe<2> u = gl_add(v[0], gl_mul(v[5], v[4], k), k);
  Fe<2> s = gl_mul(v[1], u, k);
  s = gl_add(s, gl_mul(v[3], v[4], k), k);
  s = gl_sub(s, gl_mul(v[6], v[7], k), k);
  s = gl_add(s, v[8], k);
  return gl_mul(v[2], s, k);
}

__device__ __forceinline__ Fe<2> shape_value_lazy(const Fe<2> (&v)[6], const GoldK k,
                                                  std::integral_constant<int, kShapeAbcg>) {
  const Fe<2> s = gl_add(gl_mul(gl_mul(v[0], v[1], k), v[2], k), gl_mul(v[4], v[5], k), k);
  return gl_mul(v[3], s, k);
}

// 2-limb Goldilocks shape kernels evaluate their points in lazy arithmetic: the point steps
// add a canonical difference (six ALU instructions, no compare or select), the formula's sums
// take any representatives, and the point sums are made canonical once, after the thread's
// last pair. Folds, stored tables and differences stay canonical. Measured on B200,
// plain_goldilocks n = 24: 1.60 against 1.65 ms.
#ifndef SC_GOLD_LAZY
#define SC_GOLD_LAZY 1
#endif

// Folds (if fold) and evaluates pairs q = first, first + stride, ... < last, adding the
// point sums into acc. Generic: every table's value and difference go to this block's
// [K][L][nthr] shared arrays sv / sd for eval_pair. Shape kernels keep them in registers
// (tables read in role order) and evaluate the shape's compile-time formula at each point.
// 2-limb shape kernels issue every load of a pair before its folds and run 2 blocks/SM
// (<= 128 registers for the loaded words): measured on B200, Goldilocks n = 24 went from
// 2.18 ms (loads interleaved with folds, 3 blocks/SM) to 2.01 ms.
#ifndef SC_EARLY_LOADS
#define SC_EARLY_LOADS 1
#endif

// 2-limb Goldilocks shape kernels copy each thread's next pair into shared memory with
// asynchronous copies (cp.async) while the current pair is evaluated, so its loads are in
// flight during the arithmetic instead of before it. One stage per thread, laid out
// [table][limb][thread] (16-byte entries in fold rounds, 8-byte in round 0) after the block
// reduction's scratch; the next pair's copies are issued only after every value of the
// current stage has been consumed by an arithmetic instruction, and each thread waits for its
// own copies alone (cp.async.wait_group), so no block barrier is involved.
#ifndef SC_GOLD_ASYNC
#define SC_GOLD_ASYNC 1
#endif
// The same stage for the 8-limb g(abc + de) shape kernel (SC_L8_ASYNC; 96 KB a block of 128
// threads, 2 blocks an SM) measured slower on B200: plain BLS n = 22 3.37 against 3.25 ms
// (255 registers with 120 bytes of spills, against none). Off.
#ifndef SC_L8_ASYNC
#define SC_L8_ASYNC 0
#endif
__host__ __device__ constexpr bool gold_async_stage(int L, int K, int shape) {
  return SC_GOLD_ASYNC && L == 2 && K == kFieldGoldilocks && shape != kShapeGeneric && SC_GOLD_SHAPE_FMA &&
         SC_GOLD_LAZY;
}
__host__ __device__ constexpr bool l8_async_stage(int L, int shape) { return SC_L8_ASYNC && L >= 8 && shape == kShapeAbcg; }
__host__ __device__ constexpr bool shape_async_stage(int L, int K, int shape) {
  return gold_async_stage(L, K, shape) || l8_async_stage(L, shape);
}
// Dynamic shared memory (bytes) of a compile-time shape round kernel of `threads` threads.
__host__ __device__ constexpr size_t shape_round_smem_bytes(int L, int K, int shape, int threads) {
  return 4 * (static_cast<size_t>(threads / 32) * kMaxPoints * L +
              (shape_async_stage(L, K, shape) ? static_cast<size_t>(threads) * shape_tables(shape) * L * 4 : 0));
}
__device__ __forceinline__ void cp_async_16(void* smem_dst, const void* gmem_src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_8(void* smem_dst, const void* gmem_src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
#ifndef SC_PAIR_UNROLL
#define SC_PAIR_UNROLL 1
#endif
constexpr int kPairUnroll = SC_PAIR_UNROLL;
template <int L, int K, int DMAX, int SHAPE = kShapeGeneric>
__device__ __forceinline__ void process_pairs(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                              uint64_t src_len, bool fold,
                                              const Fe<L>& r_prev, const ExprDev& E, uint32_t* sv, uint32_t* sd,
                                              uint64_t first, uint64_t last, uint64_t stride, bool skip1,
                                              Fe<L> (&acc)[DMAX + 1], const FieldParams<L, K>& F) {
  if constexpr (SHAPE != kShapeGeneric && L == 2 && K == kFieldGoldilocks && SC_GOLD_SHAPE_FMA) {
    // the shape kernels' folds and points with every Goldilocks carry on the FMA pipe
    FieldParams<2, kFieldGoldilocksFma> G;
    G.p[0] = F.p[0];
    G.p[1] = F.p[1];
    G.np = F.np;
    process_pairs<L, kFieldGoldilocksFma, DMAX, SHAPE>(src, dst, src_len, fold, r_prev, E, sv, sd, first, last, stride,
                                                        skip1, acc, G);
    return;
  }
  const int tid = threadIdx.x, nthr = blockDim.x;
  constexpr int NR = SHAPE == kShapeGeneric ? 1 : shape_tables(SHAPE);
  constexpr bool kGoldLazy = SHAPE != kShapeGeneric && L == 2 && K == kFieldGoldilocksFma && SC_GOLD_LAZY;
  constexpr bool kAsync = (kGoldLazy && SC_GOLD_ASYNC) || l8_async_stage(L, SHAPE);
  const int nv = SHAPE == kShapeGeneric ? E.num_vars : NR;
  // kAsync: this thread's stage, after the block reduction's scratch (16-byte aligned)
  uint32_t* const stage = sv + (nthr / 32) * kMaxPoints * L;
  auto issue = [&](uint64_t qn) {  // copies of pair qn into the stage
#pragma unroll
    for (int i = 0; i < NR; ++i)
#pragma unroll
      for (int l = 0; l < L; ++l) {
        const uint32_t* plane = src + (static_cast<uint64_t>(E.role[i]) * L + l) * src_len;
        const int slot = (i * L + l) * nthr + tid;
        if (fold)
          cp_async_16(reinterpret_cast<uint4*>(stage) + slot, reinterpret_cast<const uint4*>(plane) + qn);
        else
          cp_async_8(reinterpret_cast<uint2*>(stage) + slot, reinterpret_cast<const uint2*>(plane) + qn);
      }
    cp_async_commit();
  };
  if constexpr (kAsync) {
    if (first < last) issue(first);
  }
#pragma unroll(SHAPE == kShapeGeneric ? 1 : kPairUnroll)
  for (uint64_t q = first; q < last; q += stride) {
    Fe<L> sh_v[NR], sh_d[NR];
    if constexpr (kAsync) {
      cp_async_wait_all();  // this pair's copies (this thread's own) have landed
      if (fold) {
        const uint64_t dst_len = src_len >> 1;
#pragma unroll
        for (int i = 0; i < NR; ++i) {
          Fe<L> x0, x1, x2, x3;
#pragma unroll
          for (int l = 0; l < L; ++l) {
            const uint4 v = reinterpret_cast<const uint4*>(stage)[(i * L + l) * nthr + tid];
            x0.w[l] = v.x; x1.w[l] = v.y; x2.w[l] = v.z; x3.w[l] = v.w;
          }
          const Fe<L> e = fe_add(x0, fe_mul(r_prev, fe_sub(x1, x0, F), F), F);
          const Fe<L> o = fe_add(x2, fe_mul(r_prev, fe_sub(x3, x2, F), F), F);
#pragma unroll
          for (int l = 0; l < L; ++l)
            reinterpret_cast<uint2*>(dst + (static_cast<uint64_t>(E.role[i]) * L + l) * dst_len)[q] = make_uint2(e.w[l], o.w[l]);
          sh_v[i] = e;
          sh_d[i] = o;
        }
        // every value of the stage has been consumed by the folds: the next pair may land
        if (q + stride < last) issue(q + stride);
      } else {
#pragma unroll
        for (int i = 0; i < NR; ++i)
#pragma unroll
          for (int l = 0; l < L; ++l) {
            const uint2 v = reinterpret_cast<const uint2*>(stage)[(i * L + l) * nthr + tid];
            sh_v[i].w[l] = v.x;
            sh_d[i].w[l] = v.y;
          }
        // the next pair is issued after the differences below, which consume every value
      }
    } else
#if SC_EARLY_LOADS
    if constexpr (SHAPE != kShapeGeneric && L <= 2) {
      // every load of the pair first (one 16- or 8-byte load per table and limb plane), then
      // the folds: the loads of a pair are all in flight together
      if (fold) {
        uint4 raw[NR][L];
#pragma unroll
        for (int i = 0; i < NR; ++i)
#pragma unroll
          for (int l = 0; l < L; ++l)
            raw[i][l] = __ldcs(reinterpret_cast<const uint4*>(src + (static_cast<uint64_t>(E.role[i]) * L + l) * src_len) + q);
        const uint64_t dst_len = src_len >> 1;
#pragma unroll
        for (int i = 0; i < NR; ++i) {
          Fe<L> x0, x1, x2, x3;
#pragma unroll
          for (int l = 0; l < L; ++l) {
            x0.w[l] = raw[i][l].x; x1.w[l] = raw[i][l].y; x2.w[l] = raw[i][l].z; x3.w[l] = raw[i][l].w;
          }
          const Fe<L> e = fe_add(x0, fe_mul(r_prev, fe_sub(x1, x0, F), F), F);
          const Fe<L> o = fe_add(x2, fe_mul(r_prev, fe_sub(x3, x2, F), F), F);
#pragma unroll
          for (int l = 0; l < L; ++l)
            reinterpret_cast<uint2*>(dst + (static_cast<uint64_t>(E.role[i]) * L + l) * dst_len)[q] = make_uint2(e.w[l], o.w[l]);
          sh_v[i] = e;
          sh_d[i] = o;
        }
      } else {
        uint2 raw[NR][L];
#pragma unroll
        for (int i = 0; i < NR; ++i)
#pragma unroll
          for (int l = 0; l < L; ++l)
            raw[i][l] = __ldcs(reinterpret_cast<const uint2*>(src + (static_cast<uint64_t>(E.role[i]) * L + l) * src_len) + q);
#pragma unroll
        for (int i = 0; i < NR; ++i)
#pragma unroll
          for (int l = 0; l < L; ++l) {
            sh_v[i].w[l] = raw[i][l].x;
            sh_d[i].w[l] = raw[i][l].y;
          }
      }
    } else
#endif
#pragma unroll (SHAPE == kShapeGeneric ? 1 : NR)
    for (int i = 0; i < nv; ++i) {
      const int k = SHAPE == kShapeGeneric ? i : E.role[i];
      Fe<L> e, o;
      if (fold) {
        Fe<L> x0, x1, x2, x3;
#pragma unroll
        for (int l = 0; l < L; ++l) {
          const uint4 v = __ldcs(reinterpret_cast<const uint4*>(src + (static_cast<uint64_t>(k) * L + l) * src_len) + q);
          x0.w[l] = v.x; x1.w[l] = v.y; x2.w[l] = v.z; x3.w[l] = v.w;
        }
        e = fe_add(x0, fe_mul(r_prev, fe_sub(x1, x0, F), F), F);
        o = fe_add(x2, fe_mul(r_prev, fe_sub(x3, x2, F), F), F);
        const uint64_t dst_len = src_len >> 1;
#pragma unroll
        for (int l = 0; l < L; ++l)
          reinterpret_cast<uint2*>(dst + (static_cast<uint64_t>(k) * L + l) * dst_len)[q] = make_uint2(e.w[l], o.w[l]);
      } else {
#pragma unroll
        for (int l = 0; l < L; ++l) {
          const uint2 v = __ldcs(reinterpret_cast<const uint2*>(src + (static_cast<uint64_t>(k) * L + l) * src_len) + q);
          e.w[l] = v.x; o.w[l] = v.y;
        }
      }
      if constexpr (SHAPE == kShapeGeneric) {
        sm_put<L>(sv, k, tid, nthr, e);
        sm_put<L>(sd, k, tid, nthr, fe_sub(o, e, F));
      } else {
        sh_v[i] = e;
        sh_d[i] = o;  // o for now: the difference is formed below
      }
    }
    if constexpr (SHAPE == kShapeGeneric) {
      eval_pair<L, K, DMAX>(E, sv, sd, tid, nthr, skip1, acc, F);
    } else if constexpr (kGoldLazy) {
      // as below, in lazy arithmetic: sh_v / sh_d arrive canonical, the differences are
      // canonical, the stepped values and the point sums are any representatives
      constexpr int D = 4;
      static_assert(DMAX >= D, "shape kernels evaluate degree-4 shapes");
      const GoldK gk = gold_k(F);
      const std::integral_constant<int, SHAPE> shape{};
      acc[0] = gl_add(acc[0], shape_value_lazy(sh_v, gk, shape), gk);
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const Fe<L> o = sh_d[r];
        sh_d[r] = fe_sub(o, sh_v[r], F);
        sh_v[r] = o;
      }
      if constexpr (kAsync) {
        if (!fold && q + stride < last) issue(q + stride);
      }
      if (!skip1) acc[1] = gl_add(acc[1], shape_value_lazy(sh_v, gk, shape), gk);
#pragma unroll
      for (int t = 2; t <= D; ++t) {
#pragma unroll
        for (int r = 0; r < NR; ++r) sh_v[r] = gl_add_c(sh_v[r], sh_d[r], gk);
        acc[t] = gl_add(acc[t], shape_value_lazy(sh_v, gk, shape), gk);
      }
    } else {
      // point 0: e; point 1: o (skipped when skip1); then v(t) = v(t - 1) + (o - e)
      constexpr int D = 4;
      static_assert(DMAX >= D, "shape kernels evaluate degree-4 shapes");
      acc[0] = fe_add(acc[0], shape_value<L, K>(sh_v, F, std::integral_constant<int, SHAPE>{}), F);
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const Fe<L> o = sh_d[r];
        sh_d[r] = fe_sub(o, sh_v[r], F);
        sh_v[r] = o;
      }
      if constexpr (kAsync) {
        if (!fold && q + stride < last) issue(q + stride);
      }
      if (!skip1) acc[1] = fe_add(acc[1], shape_value<L, K>(sh_v, F, std::integral_constant<int, SHAPE>{}), F);
#pragma unroll
      for (int t = 2; t <= D; ++t) {
#pragma unroll
        for (int r = 0; r < NR; ++r) sh_v[r] = fe_add(sh_v[r], sh_d[r], F);
        acc[t] = fe_add(acc[t], shape_value<L, K>(sh_v, F, std::integral_constant<int, SHAPE>{}), F);
      }
    }
  }
  if constexpr (kGoldLazy || lazy_generic<L, K>()) {
    const GoldK gk = gold_k(F);
#pragma unroll
    for (int t = 0; t <= DMAX; ++t) acc[t] = gl_canon(acc[t], gk);
  }
}

// Reduce acc[0..d] over the block; the block sums land in red_out[t * L + l] (shared).
template <int L, int K, int N>
__device__ __forceinline__ void block_reduce(Fe<L> (&acc)[N], int d, uint32_t* scratch, uint32_t* red_out,
                                             const FieldParams<L, K>& F) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
#pragma unroll
  for (int t = 0; t < N; ++t) {
    if (t > d) break;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc[t] = fe_add(acc[t], fe_shfl_down(acc[t], off), F);
  }
  if (lane == 0) {
#pragma unroll
    for (int t = 0; t < N; ++t) {
      if (t > d) break;
      st_fe<L>(scratch + (warp * kMaxPoints + t) * L, acc[t]);
    }
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int t = 0; t < N; ++t) {
      if (t > d) break;
      Fe<L> v = lane < nwarps ? ld_fe<L>(scratch + (lane * kMaxPoints + t) * L) : fe_zero<L>();
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v = fe_add(v, fe_shfl_down(v, off), F);
      if (lane == 0) st_fe<L>(red_out + t * L, v);
    }
  }
  __syncthreads();
}

// Sums the partials of blocks/items [first, first + count) into g_sm[t * L + l] (block-wide).
template <int L, int K, int N>
__device__ __forceinline__ void reduce_partials(const uint32_t* partials, uint64_t first, uint64_t count, int d,
                                                uint32_t* scratch, uint32_t* g_sm, const FieldParams<L, K>& F) {
  Fe<L> acc[N];
#pragma unroll
  for (int t = 0; t < N; ++t) acc[t] = fe_zero<L>();
  for (uint64_t b = threadIdx.x; b < count; b += blockDim.x) {
    const uint32_t* pb = partials + (first + b) * kMaxPoints * L;
#pragma unroll
    for (int t = 0; t < N; ++t) {
      if (t > d) break;
      acc[t] = fe_add(acc[t], ld_fe_cg<L>(pb + t * L), F);
    }
  }
  block_reduce<L, K, N>(acc, d, scratch, g_sm, F);
}

template <int L>
__device__ __forceinline__ Fe<L> fc_get(const uint32_t* row) {
  return ld_fe<L>(row);
}

// g(r) for the polynomial with values g_sm[t] at t = 0..d (Lagrange form with the field's
// precomputed weights); lane t < d + 1 forms one term, the warp sums them (all lanes call).
template <int L, int K>
__device__ __forceinline__ Fe<L> lagrange_at(const uint32_t* g_sm, int d, const Fe<L>& r, const FieldConsts& fc,
                                             const FieldParams<L, K>& F) {
  const int lane = threadIdx.x & 31;
  Fe<L> term = fe_zero<L>();
  if (lane <= d) {
    term = fe_mul(ld_fe<L>(g_sm + lane * L), fc_get<L>(fc.lag[d][lane]), F);
    for (int s = 0; s <= d; ++s)
      if (s != lane) term = fe_mul(term, fe_sub(r, fc_get<L>(fc.pts[s]), F), F);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) term = fe_add(term, fe_shfl_down(term, off), F);
  return fe_shfl(term, 0);
}

// Last block of a round: g_j is in g_sm[t * L + l] (point 1 still empty when skip1).
// Warp 0 does all of this.
template <int L, int K>
__device__ void finalize_round(const RoundArgs& A, const ExprDev& E, const FieldParams<L, K>& F, uint32_t* g_sm,
                               uint8_t* msg) {
  const int lane = threadIdx.x & 31;
  const int d = E.degree;
  const int j = A.round;
  const FieldConsts& fc = *A.fc;
  // 0. g(1) from the claim this round must meet, or, when asked, that claim checked
  if (A.skip1) {
    if (lane == 0) st_fe<L>(g_sm + L, fe_sub(ld_fe_cg<L>(A.st.claim), ld_fe<L>(g_sm), F));
    __syncwarp();
  } else if (A.check_claim && lane == 0) {
    const Fe<L> s = fe_add(ld_fe<L>(g_sm), ld_fe<L>(g_sm + L), F);
    const Fe<L> c = ld_fe_cg<L>(A.st.claim);
    bool eq = true;
#pragma unroll
    for (int l = 0; l < L; ++l) eq = eq && s.w[l] == c.w[l];
    if (!eq) atomicOr(A.st.status, kStatusClaim);
  }
  // 1. round polynomial and checksum
  for (int i = lane; i < (d + 1) * L; i += 32) A.st.polys[(j * kMaxPoints + i / L) * L + i % L] = g_sm[i];
  if (lane == 0) {
    uint64_t cs = 0;
    for (int t = 0; t <= d; ++t)
      for (int l = 0; l < L; ++l) cs += static_cast<uint64_t>(l + 1) * g_sm[t * L + l];
    *A.st.checksum += cs;
    if (j == 0) {
      const Fe<L> c0 = fe_add(ld_fe<L>(g_sm), ld_fe<L>(g_sm + L), F);
      st_fe<L>(A.st.claim0, c0);
    }
  }
  // 2. challenge r_j
  Fe<L> r;
  if (A.mode == kChallengeSha3) {
    const char dom[] = "zkduel:field-sweep:v1";
    constexpr int kDom = sizeof(dom) - 1;
    const int nwords = 1 + (d + 1) * L;
    if (lane < kDom) msg[lane] = static_cast<uint8_t>(dom[lane]);
    for (int i = lane; i < nwords; i += 32) {
      const uint32_t w = i == 0 ? static_cast<uint32_t>(j) : g_sm[i - 1];
      msg[kDom + 4 * i + 0] = static_cast<uint8_t>(w);
      msg[kDom + 4 * i + 1] = static_cast<uint8_t>(w >> 8);
      msg[kDom + 4 * i + 2] = static_cast<uint8_t>(w >> 16);
      msg[kDom + 4 * i + 3] = static_cast<uint8_t>(w >> 24);
    }
    __syncwarp();
    uint32_t dig[8];
    sha3_256_warp(msg, kDom + 4 * nwords, dig);
    // digest (little-endian 256-bit D) -> D R mod p = sum_i (w_i mod p) * R^2 2^(32 i) / R
    Fe<L> term = fe_zero<L>();
    if (lane < 8) {
      uint32_t w = dig[0];
#pragma unroll
      for (int i = 1; i < 8; ++i)
        if (lane == i) w = dig[i];
      if (fc.p_small) w %= fc.p_small;
      Fe<L> wf = fe_zero<L>();
      wf.w[0] = w;
      term = fe_mul(wf, fc_get<L>(fc.kdig[lane]), F);
    }
#pragma unroll
    for (int off = 4; off > 0; off >>= 1) term = fe_add(term, fe_shfl_down(term, off), F);
    r = fe_shfl(term, 0);
    if (lane == 0) st_fe<L>(A.st.chals + j * L, r);
  } else if (A.mode == kChallengeFixed) {
    r = fc_get<L>(fc.one);
    if (lane == 0) st_fe<L>(A.st.chals + j * L, r);
  } else {
    r = ld_fe_cg<L>(A.st.chals + j * L);
  }
  // 3. g_j(r_j): the next round's claim, and in the last round the final claim
  const bool last_round = j == A.num_rounds - 1;
  if (A.want_claim || last_round) {
    const Fe<L> gr = lagrange_at<L, K>(g_sm, d, r, fc, F);
    if (lane == 0) st_fe<L>(last_round ? A.st.finals : A.st.claim, gr);
  }
  // 4. last round: f_k(r) per table
  if (last_round) {
    const uint32_t* tab = A.fold ? A.dst : A.src;  // T_{n-1}: 2 entries per plane
    for (int k = lane; k < E.num_vars; k += 32) {
      Fe<L> e, o;
#pragma unroll
      for (int l = 0; l < L; ++l) {
        e.w[l] = __ldcg(tab + (k * L + l) * 2 + 0);
        o.w[l] = __ldcg(tab + (k * L + l) * 2 + 1);
      }
      const Fe<L> f = fe_add(e, fe_mul(r, fe_sub(o, e, F), F), F);
      st_fe<L>(A.st.finals + (1 + k) * L, f);
    }
  }
}

// Dynamic shared memory per thread: values and differences of every table.
__host__ __device__ constexpr int round_smem_words_per_thread(int K, int L) { return 2 * K * L; }

// Launch shape per limb count: 8-limb kernels hold (DMAX + 1) x 8-word point arrays per
// thread, so they run 128-thread blocks and ask the compiler for at least 3 blocks per SM
// (<= 168 registers; on B200 the mixed 512-proof stream ran 10% slower with 2 or 4 blocks
// with the C++ product, 5% and 4% slower with the even/odd product); smaller fields run
// 256-thread blocks.
__host__ __device__ constexpr int kernel_threads(int L) { return L >= 8 ? 128 : 256; }
#ifndef SC_PP_MIN_LIMBS
#define SC_PP_MIN_LIMBS 8
#endif
// Fields of at least this many limbs evaluate generic expressions point-parallel
// (prover_pp.cuh) in the plain round kernel.
__host__ __device__ constexpr bool use_point_parallel(int L) { return L >= SC_PP_MIN_LIMBS; }
constexpr int kPointParallelThreads = 128;
#ifndef SC_L8_MIN_BLOCKS
#define SC_L8_MIN_BLOCKS 3
#endif
// 4-limb kernels at 2 blocks/SM (<= 128 registers: 16 warps instead of 8; the degree <= 7
// class spills 36 bytes). Measured on B200 over 4,000 requests of the served stream (2^127 - 1)
// at 80% load: p50 1.34 -> 1.04 ms, p90 13.0 -> 6.6 ms, p99 39-43 -> 23.3 ms; the plain 4-limb
// proofs took the same time either way.
#ifndef SC_L4_MIN_BLOCKS
#define SC_L4_MIN_BLOCKS 2
#endif
// 2-limb generic and batched kernels at 3 blocks/SM (<= 85 registers; 74-80 used, the
// degree <= 7 class spills 4-20 bytes): the 512-proof mixed stream went from 9.89k to 10.16k
// proofs/s (the 64-bit ticks' busy time 31.5 -> 30.0 ms), plain 64-bit proofs the same. At 4
// limbs, 3 blocks/SM spilled 700+ bytes and served p50 went from 1.03 to 1.31 ms.
#ifndef SC_L2_MIN_BLOCKS
#define SC_L2_MIN_BLOCKS 3
#endif
__host__ __device__ constexpr int kernel_min_blocks(int L) {
  return L >= 8 ? SC_L8_MIN_BLOCKS : (L == 4 ? SC_L4_MIN_BLOCKS : (L == 2 ? SC_L2_MIN_BLOCKS : 1));
}
#ifndef SC_SHAPE_MIN_BLOCKS
#define SC_SHAPE_MIN_BLOCKS 2
#endif
// Shape kernels of the 1- and 2-limb fields are memory-bound: ask for more resident blocks.
// The 8-limb shape kernels hold every table's value and difference in registers: at 3 blocks
// of 128 threads they spilled; at 2 (no spills) plain BLS n = 22 took 3.28 against 3.37 ms
// with the even/odd product (the batched 8-limb kernels stay at 3, where 2 was 5% slower).
#ifndef SC_SHAPE_L8_MIN_BLOCKS
#define SC_SHAPE_L8_MIN_BLOCKS 2
#endif
// The batched kernel per limb count and degree class: the 8-limb classes of degree 6-7 hold
// 7-8 points of 8-limb accumulators and products in registers.
#ifndef SC_BATCH_L8_HIGH_MIN_BLOCKS
#define SC_BATCH_L8_HIGH_MIN_BLOCKS SC_L8_MIN_BLOCKS
#endif
#ifndef SC_BATCH_L8_HIGH_DMAX
#define SC_BATCH_L8_HIGH_DMAX 6
#endif
__host__ __device__ constexpr int batch_min_blocks(int L, int dmax) {
  return (L >= 8 && dmax >= SC_BATCH_L8_HIGH_DMAX) ? SC_BATCH_L8_HIGH_MIN_BLOCKS : kernel_min_blocks(L);
}
__host__ __device__ constexpr int round_min_blocks(int L, int shape) {
  return (shape != 0 && L <= 2) ? SC_SHAPE_MIN_BLOCKS
                                : ((shape != 0 && L >= 8) ? SC_SHAPE_L8_MIN_BLOCKS : kernel_min_blocks(L));
}

template <int L, int K, int DMAX, int SHAPE = kShapeGeneric>
__global__ void __launch_bounds__(kernel_threads(L), round_min_blocks(L, SHAPE))
    round_kernel(const RoundArgs A, const ExprDev E, const FieldParams<L, K> F) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ __align__(16) uint32_t g_sm[kMaxPoints * kMaxLimbs];
  __shared__ __align__(16) uint8_t msg[3 * 136];
  __shared__ int is_last;

  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int d = E.degree;
  uint32_t* sv = smem;                           // [K][L][nthr] values at the current point
  uint32_t* sd = smem + E.num_vars * L * nthr;   // [K][L][nthr] differences o - e

  Fe<L> acc[DMAX + 1];
#pragma unroll
  for (int t = 0; t <= DMAX; ++t) acc[t] = fe_zero<L>();
  Fe<L> r_prev = fe_zero<L>();
  if (A.fold) r_prev = ld_fe_cg<L>(A.st.chals + (A.round - 1) * L);
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * nthr;
  process_pairs<L, K, DMAX, SHAPE>(A.src, A.dst, A.src_len, A.fold != 0, r_prev, E, sv, sd,
                                   static_cast<uint64_t>(blockIdx.x) * nthr + tid, A.pairs, stride, A.skip1 != 0, acc, F);

  // block partial -> global; the last block reduces all partials
  __syncthreads();
  block_reduce<L, K, DMAX + 1>(acc, d, smem, g_sm, F);
  for (int i = tid; i < (d + 1) * L; i += nthr) A.partials[static_cast<uint64_t>(blockIdx.x) * kMaxPoints * L + i] = g_sm[i];
  __threadfence();
  __syncthreads();
  if (tid == 0) is_last = (atomicAdd(A.st.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  reduce_partials<L, K, DMAX + 1>(A.partials, 0, gridDim.x, d, smem, g_sm, F);
  if (A.ext_out) {
    for (int i = tid; i < (d + 1) * L; i += nthr) A.ext_out[i] = g_sm[i];
  } else if (tid < 32) {
    finalize_round<L, K>(A, E, F, g_sm, msg);
  }
  if (tid == 0) {
    __threadfence();
    *A.st.counter = 0;
  }
}

// ------------------------------------------------------------------------------ resume folds
//
// T_i = T_{i-1} + r_{i-1} (odd - even) and nothing else: the folds that bring a resumed
// proof's tables to the round it continues from (the round kernel folds the last one
// itself). One thread per output pair of one table: a 16-byte load per limb plane in, an
// 8-byte store per plane out, as the round kernel's fused fold. src_len >= 4 entries.
template <int L, int K>
__global__ void __launch_bounds__(256) fold_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                                   uint64_t src_len, int num_tables, const uint32_t* r_dev,
                                                   const FieldParams<L, K> F) {
  const uint64_t quads = src_len >> 2;  // output pairs per table
  const uint64_t total = quads * static_cast<uint64_t>(num_tables);
  const uint64_t dst_len = src_len >> 1;
  const Fe<L> r = ld_fe_cg<L>(r_dev);
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t k = i / quads, q = i - k * quads;
    Fe<L> x0, x1, x2, x3;
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const uint4 v = __ldcs(reinterpret_cast<const uint4*>(src + (k * L + l) * src_len) + q);
      x0.w[l] = v.x; x1.w[l] = v.y; x2.w[l] = v.z; x3.w[l] = v.w;
    }
    const Fe<L> e = fe_add(x0, fe_mul(r, fe_sub(x1, x0, F), F), F);
    const Fe<L> o = fe_add(x2, fe_mul(r, fe_sub(x3, x2, F), F), F);
#pragma unroll
    for (int l = 0; l < L; ++l) reinterpret_cast<uint2*>(dst + (k * L + l) * dst_len)[q] = make_uint2(e.w[l], o.w[l]);
  }
}

// ------------------------------------------------------------------------------ batched
//
// Many independent proofs advance together, one launch per "tick" and degree class: a
// persistent kernel whose blocks pull (proof round, tile of pairs) items from a device work
// queue (an atomic counter over the tick's item list). Every item leaves one partial in its
// round's partial slots; the block that finishes the last item of a proof's round (per-proof
// atomic ticket) reduces that round's partials and finalises it -- SHA3 challenge included --
// while the other blocks go on with other proofs' items. A round's items may be spread over
// several ticks (the served prover slices large rounds): the ticket counts to the round's
// item total, whichever tick its last item runs in.
//
// Tail rounds: once a proof's round fits in one item, the block that proves it also proves
// every later round of that proof (tail_rounds of them), one after another with block
// barriers in between -- a few microseconds a round instead of one tick each. Round j + 1
// reads T_j, which this block wrote itself, and r_j, which its warp 0 just derived.

struct BatchRound {
  RoundArgs args;        // this proof's round (src/dst/len/pairs/round/fold/mode/flags/fc/state)
  const ExprDev* expr;   // this proof's expression
  uint32_t* partials;    // the round's partial slots: [round_items][kMaxPoints][L]
  int32_t first_item;    // this tick's items of the round: [first_item, first_item + num_items)
  int32_t num_items;
  int32_t item_base;     // round-relative index of this tick's first item of the round
  int32_t round_items;   // items of the whole round, over all ticks
  int32_t tail_rounds;   // > 0: the block that finalises this round proves the next tail_rounds too
  uint32_t skip1_min_pairs;  // tail rounds: g(1) from the claim when a round has this many pairs
  uint32_t* fold_a;      // tail rounds: T_i for odd i
  uint32_t* fold_b;      //              T_i for even i >= 2
};

struct BatchItem {
  int32_t round;       // index into the tick's BatchRound array
  int32_t pad;
  uint64_t start;      // pairs [start, start + count)
  uint64_t count;
};

struct BatchTickArgs {
  const BatchRound* rounds;
  const BatchItem* items;  // nullptr: one round, item i = pairs [i tile, (i + 1) tile)
  int32_t num_items;
  int32_t pad;
  uint32_t* head;          // queue counter of this tick (zero before the launch); nullptr:
                           // block b does item b alone (grid = num_items)
  uint64_t tile;           // pairs per item when items is nullptr
};

template <int L, int K, int DMAX>
__global__ void __launch_bounds__(kernel_threads(L), batch_min_blocks(L, DMAX))
    batch_round_kernel(const BatchTickArgs T, const FieldParams<L, K> F) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ __align__(16) uint32_t g_sm[kMaxPoints * kMaxLimbs];
  __shared__ __align__(16) uint8_t msg[3 * 136];
  __shared__ __align__(16) ExprDev E;
  __shared__ __align__(16) BatchRound R;
  __shared__ const ExprDev* cur_expr;
  __shared__ int item_sm, is_last;

  const int tid = threadIdx.x, nthr = blockDim.x;
  if (tid == 0) cur_expr = nullptr;
  for (int pass = 0;; ++pass) {
    __syncthreads();
    if (tid == 0)
      item_sm = T.head ? static_cast<int>(atomicAdd(T.head, 1u)) : (pass == 0 ? static_cast<int>(blockIdx.x) : T.num_items);
    __syncthreads();
    const int it = item_sm;
    if (it >= T.num_items) break;
    BatchItem I;
    if (T.items) {
      I = T.items[it];
    } else {
      I.round = 0;
      I.start = static_cast<uint64_t>(it) * T.tile;
    }
    if (tid == 0) R = T.rounds[I.round];
    __syncthreads();
    if (!T.items) I.count = R.args.pairs - I.start < T.tile ? R.args.pairs - I.start : T.tile;
    if (R.expr != cur_expr) {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(R.expr);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&E);
      for (int i = tid; i < static_cast<int>(sizeof(ExprDev) / 4); i += nthr) dst[i] = src[i];
      __syncthreads();
      if (tid == 0) cur_expr = R.expr;
    }
    const int d = E.degree;
    uint32_t* sv = smem;
    uint32_t* sd = smem + E.num_vars * L * nthr;
    // k = 0: this item of the proof's round; k >= 1: the proof's tail rounds (only in the
    // block that finalised round k - 1; R.args then describes round R.args.round)
    for (int k = 0;; ++k) {
      Fe<L> acc[DMAX + 1];
#pragma unroll
      for (int t = 0; t <= DMAX; ++t) acc[t] = fe_zero<L>();
      Fe<L> r_prev = fe_zero<L>();
      if (R.args.fold) r_prev = ld_fe_cg<L>(R.args.st.chals + (R.args.round - 1) * L);
      const uint64_t q0 = k == 0 ? I.start : 0, q1 = k == 0 ? I.start + I.count : R.args.pairs;
      process_pairs<L, K, DMAX>(R.args.src, R.args.dst, R.args.src_len, R.args.fold != 0, r_prev, E, sv, sd, q0 + tid,
                                q1, nthr, R.args.skip1 != 0, acc, F);
      __syncthreads();
      block_reduce<L, K, DMAX + 1>(acc, d, smem, g_sm, F);
      if (k == 0) {
        uint32_t* slot = R.partials + static_cast<uint64_t>(R.item_base + (it - R.first_item)) * kMaxPoints * L;
        for (int i = tid; i < (d + 1) * L; i += nthr) slot[i] = g_sm[i];
        __threadfence();
        __syncthreads();
        if (tid == 0) is_last = (atomicAdd(R.args.st.counter, 1u) == static_cast<uint32_t>(R.round_items - 1));
        __syncthreads();
        if (!is_last) break;
        __threadfence();
        reduce_partials<L, K, DMAX + 1>(R.partials, 0, R.round_items, d, smem, g_sm, F);
      }
      if (tid < 32) finalize_round<L, K>(R.args, E, F, g_sm, msg);
      if (k == 0 && tid == 0) {
        __threadfence();
        *R.args.st.counter = 0;
      }
      if (k == R.tail_rounds) break;
      __syncthreads();  // the finalisation read R.args; r_j and T_j are visible to the block
      if (tid == 0) {   // round j + 1 of the same proof
        RoundArgs& A = R.args;
        const int j = A.round + 1;
        if (j >= 2) A.src = A.dst;  // T_j (round 1 folds the tables themselves)
        A.dst = (j & 1) ? R.fold_a : R.fold_b;
        A.round = j;
        A.pairs >>= 1;
        A.src_len = A.pairs * 4;
        A.fold = 1;
        A.skip1 = A.pairs >= R.skip1_min_pairs ? 1 : 0;
        A.want_claim = (j + 1 < A.num_rounds && (A.pairs >> 1) >= R.skip1_min_pairs) ? 1 : 0;
        A.check_claim = 0;
      }
      __syncthreads();
    }
  }
}

}  // namespace sc
