// Point-parallel evaluation of a round: one pair per group of G lanes, one point per lane.
//
// The register-array evaluator (prover.cuh, eval_pair) gives each thread whole pairs: it holds
// the d+1 point products and point sums of a pair, (DMAX + 1) x L words each. At 8 limbs that
// is up to 128 registers before any product runs, so only 12 warps fit on an SM and the
// dependent multiply-add chains of the Montgomery products stall the schedulers ("wait").
//
// Here a pair belongs to a group of G lanes (G = 2, 4 or 8: the power of two >= the number of
// points the round evaluates). Lane i of the group evaluates point pts[i] (0, then 1 unless
// g(1) comes from the claim, then 2..d); lanes past the last point idle in the evaluation.
//   1. load / fold: the group's lanes split the tables (lane i takes tables i, i + G, ...),
//      fold them with r_{j-1} (two products a table), write T_j, and put every table's value e
//      and difference o - e into the pair's shared-memory slot;
//   2. evaluate: each lane computes the expression at its point from the slot: a factor's value
//      at p is e + p (o - e), p (o - e) by an addition chain (p <= 7), and one product per
//      factor after the first;
//   3. reduce: each lane keeps one point sum; lanes with the same point are summed across the
//      warp (shuffles over the pair index) and across warps (shared memory).
// A lane holds one sum, one product and one factor, so the 8-limb kernel fits 4 x 128 threads
// per SM, and a round's pairs spread over many more blocks. Results are bit-identical to the
// register-array evaluator (same arithmetic, exact).
//
// Measured on B200 (the mixed 512-proof stream): proving one 256-bit proof at a time, this
// kernel is 18% faster than the register-array one (small rounds reach more SMs); inside the
// batched ticks, where many proofs already fill the GPU, it was 25% slower (more products --
// no extrapolated terms -- and per-lane point stepping), so batches keep the register arrays.
#pragma once
#include "prover.cuh"

namespace sc {

// Points a round evaluates, in lane order, and the lane-group size.
struct PointPlan {
  int npts;   // points evaluated
  int G;      // lanes per pair: power of two >= npts
  int pts[kMaxPoints];
};

__device__ __forceinline__ PointPlan point_plan(int d, bool skip1) {
  PointPlan P;
  P.npts = 0;
  for (int t = 0; t <= d; ++t)
    if (!(skip1 && t == 1)) P.pts[P.npts++] = t;
  P.G = P.npts <= 1 ? 1 : (P.npts <= 2 ? 2 : (P.npts <= 4 ? 4 : 8));
  return P;
}

// Shared-memory words a block of `threads` lanes gets: pair slots for groups of 2 lanes and up
// to kmax tables (a slot is 2 kmax L words; a round with 1-lane groups uses the slots it has,
// the other lanes idle), and at least the reduction scratch, which reuses them.
__host__ __device__ constexpr int pp_smem_words(int threads, int kmax, int L) {
  return (threads / 2) * 2 * kmax * L > (threads / 32) * kMaxPoints * L ? (threads / 2) * 2 * kmax * L
                                                                         : (threads / 32) * kMaxPoints * L;
}

// Pairs a block holds at once: one per group, as far as the dynamic shared memory goes.
template <int L>
__device__ __forceinline__ int pp_slots(const PointPlan& P, int nv) {
  uint32_t dyn_bytes;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn_bytes));
  const int cap = static_cast<int>(dyn_bytes / 4) / (2 * nv * L);
  const int want = static_cast<int>(blockDim.x) / P.G;
  return want < cap ? want : cap;
}

// x * c for a small non-negative c (<= 7), by doubling and adding.
template <int L, int K>
__device__ __forceinline__ Fe<L> fe_times_small(const Fe<L>& x, int c, const FieldParams<L, K>& F) {
  Fe<L> acc = fe_zero<L>();
  Fe<L> base = x;
  bool any = false;
  for (int b = 0; b < 3; ++b) {
    if (c & (1 << b)) {
      acc = any ? fe_add(acc, base, F) : base;
      any = true;
    }
    if (b < 2 && (c >> (b + 1))) base = fe_add(base, base, F);
  }
  return acc;
}

// The expression at point p from a pair's slot (e[k], d[k] for every table k).
template <int L, int K>
__device__ __forceinline__ Fe<L> pp_eval_point(const ExprDev& E, const uint32_t* slot_e, const uint32_t* slot_d,
                                               int p, const FieldParams<L, K>& F) {
  auto value = [&](int k) {
    Fe<L> e, d;
#pragma unroll
    for (int l = 0; l < L; ++l) {
      e.w[l] = slot_e[k * L + l];
      d.w[l] = slot_d[k * L + l];
    }
    return p == 0 ? e : fe_add(e, fe_times_small(d, p, F), F);
  };
  Fe<L> acc = fe_zero<L>();
  for (int i = 0; i < E.num_terms; ++i) {
    const int off = E.term_off[i];
    const int len = E.term_len[i];
    const int kind = E.coeff_kind[i];
    Fe<L> prod = value(E.flat[off]);
    if (kind == kCoeffSmall) {
      const int32_t c = E.coeff_small[i];
      prod = fe_mul_small(prod, c < 0 ? static_cast<uint32_t>(-static_cast<int64_t>(c)) : static_cast<uint32_t>(c), F);
    } else if (kind == kCoeffMont) {
      Fe<L> cm;
#pragma unroll
      for (int l = 0; l < L; ++l) cm.w[l] = E.coeff_mont[i][l];
      prod = fe_mul(prod, cm, F);
    }
    for (int f = 1; f < len; ++f) prod = fe_mul(prod, value(E.flat[off + f]), F);
    const bool neg = kind == kCoeffMinus || (kind == kCoeffSmall && E.coeff_small[i] < 0);
    acc = neg ? fe_sub(acc, prod, F) : fe_add(acc, prod, F);
  }
  return acc;
}

// Pairs first, first + stride, ... (each base pair and the slots - 1 after it) below `last`:
// folded if `fold`, evaluated point-parallel into `acc` (this lane's point sum). Every lane of
// the block calls it with the same arguments; slots = pp_slots().
template <int L, int K>
__device__ __forceinline__ void pp_process_pairs(const uint32_t* src, uint32_t* dst, uint64_t src_len, bool fold,
                                                 const Fe<L>& r_prev, const ExprDev& E, const PointPlan& P,
                                                 uint32_t* smem, int slots, uint64_t first, uint64_t last,
                                                 uint64_t stride, Fe<L>& acc, const FieldParams<L, K>& F) {
  const int tid = threadIdx.x;
  const int G = P.G;
  const int slot = tid / G;     // this lane's pair slot in the block (a group never spans warps)
  const int gi = tid % G;       // lane within the group
  const int nv = E.num_vars;
  uint32_t* se = smem + static_cast<size_t>(slot) * 2 * nv * L;
  uint32_t* sd = se + nv * L;
  const int my_point = gi < P.npts ? P.pts[gi] : -1;
  for (uint64_t base = first; base < last; base += stride) {
    const uint64_t q = base + slot;
    const bool active = slot < slots && q < last;
    if (active) {
      for (int k = gi; k < nv; k += G) {
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
        const Fe<L> d = fe_sub(o, e, F);
#pragma unroll
        for (int l = 0; l < L; ++l) {
          se[k * L + l] = e.w[l];
          sd[k * L + l] = d.w[l];
        }
      }
    }
    __syncwarp();
    if (active && my_point >= 0) acc = fe_add(acc, pp_eval_point<L, K>(E, se, sd, my_point, F), F);
    __syncwarp();
  }
}

// Block sum of every point: lane gi of each group holds point pts[gi]. The sums land in
// red_out[t * L + l] for t = 0..d (zero for point 1 when it was not evaluated).
template <int L, int K>
__device__ __forceinline__ void pp_block_reduce(Fe<L> acc, const PointPlan& P, int d, uint32_t* scratch,
                                                uint32_t* red_out, const FieldParams<L, K>& F) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const int G = P.G;
  // sum over the groups of the warp (lanes with equal lane % G)
  for (int off = 16; off >= G; off >>= 1) acc = fe_add(acc, fe_shfl_down(acc, off), F);
  __syncthreads();  // the pair slots are free again
  // zero, then this warp's point sums (point 1 under skip1 and points past d stay zero)
  if (lane < kMaxPoints) st_fe<L>(scratch + (warp * kMaxPoints + lane) * L, fe_zero<L>());
  __syncwarp();
  if (lane < G && lane < P.npts) st_fe<L>(scratch + (warp * kMaxPoints + P.pts[lane]) * L, acc);
  __syncthreads();
  if (warp == 0) {
    for (int t = 0; t <= d; ++t) {
      Fe<L> v = lane < nwarps ? ld_fe<L>(scratch + (lane * kMaxPoints + t) * L) : fe_zero<L>();
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v = fe_add(v, fe_shfl_down(v, off), F);
      if (lane == 0) st_fe<L>(red_out + t * L, v);
    }
  }
  __syncthreads();
}

// Sums partial slots [0, count) into g_sm[t * L + l], one point at a time (one accumulator
// per lane); block-wide.
template <int L, int K>
__device__ __forceinline__ void pp_reduce_partials(const uint32_t* partials, uint64_t count, int d, uint32_t* scratch,
                                                   uint32_t* g_sm, const FieldParams<L, K>& F) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  for (int t = 0; t <= d; ++t) {
    Fe<L> acc = fe_zero<L>();
    for (uint64_t b = tid; b < count; b += blockDim.x) acc = fe_add(acc, ld_fe_cg<L>(partials + (b * kMaxPoints + t) * L), F);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc = fe_add(acc, fe_shfl_down(acc, off), F);
    if (lane == 0) st_fe<L>(scratch + warp * L, acc);
    __syncthreads();
    if (warp == 0) {
      Fe<L> v = lane < nwarps ? ld_fe<L>(scratch + lane * L) : fe_zero<L>();
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v = fe_add(v, fe_shfl_down(v, off), F);
      if (lane == 0) st_fe<L>(g_sm + t * L, v);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------ kernels

template <int L, int K>
__global__ void __launch_bounds__(128, 4) round_kernel_pp(const RoundArgs A, const ExprDev E, const FieldParams<L, K> F) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ __align__(16) uint32_t g_sm[kMaxPoints * kMaxLimbs];
  __shared__ __align__(16) uint8_t msg[3 * 136];
  __shared__ int is_last;
  const int tid = threadIdx.x;
  const int d = E.degree;
  const PointPlan P = point_plan(d, A.skip1 != 0);
  Fe<L> acc = fe_zero<L>();
  Fe<L> r_prev = fe_zero<L>();
  if (A.fold) r_prev = ld_fe_cg<L>(A.st.chals + (A.round - 1) * L);
  const int slots = pp_slots<L>(P, E.num_vars);
  pp_process_pairs<L, K>(A.src, A.dst, A.src_len, A.fold != 0, r_prev, E, P, smem, slots,
                         static_cast<uint64_t>(blockIdx.x) * slots, A.pairs,
                         static_cast<uint64_t>(slots) * gridDim.x, acc, F);
  pp_block_reduce<L, K>(acc, P, d, smem, g_sm, F);
  for (int i = tid; i < (d + 1) * L; i += blockDim.x)
    A.partials[static_cast<uint64_t>(blockIdx.x) * kMaxPoints * L + i] = g_sm[i];
  __threadfence();
  __syncthreads();
  if (tid == 0) is_last = (atomicAdd(A.st.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  pp_reduce_partials<L, K>(A.partials, gridDim.x, d, smem, g_sm, F);
  if (A.ext_out) {
    for (int i = tid; i < (d + 1) * L; i += blockDim.x) A.ext_out[i] = g_sm[i];
  } else if (tid < 32) {
    finalize_round<L, K>(A, E, F, g_sm, msg);
  }
  if (tid == 0) {
    __threadfence();
    *A.st.counter = 0;
  }
}

}  // namespace sc
