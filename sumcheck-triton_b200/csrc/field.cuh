// Field elements and their arithmetic on the device.
//
// An element of a field with L 32-bit limbs is Fe<L>: little-endian limbs, Montgomery form
// (x R mod p, R = 2^(32 L)), always fully reduced (< p). Fully reduced Montgomery limbs are
// unique, so they are what the transcript hashes and the checksum sums, exactly as in the
// reference (cuda/src/field_sumcheck.cu:1046-1049, :857-907).
//
// The carry chains themselves are inline PTX in field_ptx.cuh (generated).
#pragma once
#include <cstdint>

#include "field_ptx.cuh"

namespace sc {

constexpr int kMaxLimbs = 8;
constexpr int kMaxPoints = 8;  // t = 0..7, degree <= 7

template <int L>
struct Fe {
  uint32_t w[L];
};

// The two constants every product needs. Passed by value as a kernel parameter, so it
// lives in the constant bank and the multiply-adds read it from there.
template <int L>
struct FieldParams {
  uint32_t p[L];
  uint32_t np;  // -p^-1 mod 2^32
};

template <int L>
__device__ __forceinline__ Fe<L> fe_zero() {
  Fe<L> z;
#pragma unroll
  for (int i = 0; i < L; ++i) z.w[i] = 0;
  return z;
}

template <int L>
__device__ __forceinline__ Fe<L> fe_add(const Fe<L>& a, const Fe<L>& b, const FieldParams<L>& F) {
  Fe<L> r;
  ptx_add_mod<L>(r.w, a.w, b.w, F.p);
  return r;
}

template <int L>
__device__ __forceinline__ Fe<L> fe_sub(const Fe<L>& a, const Fe<L>& b, const FieldParams<L>& F) {
  Fe<L> r;
  ptx_sub_mod<L>(r.w, a.w, b.w, F.p);
  return r;
}

template <int L>
__device__ __forceinline__ Fe<L> fe_mul(const Fe<L>& a, const Fe<L>& b, const FieldParams<L>& F) {
  Fe<L> r;
  ptx_mont_mul<L>(r.w, a.w, b.w, F.p, F.np);
  return r;
}

template <int L>
__device__ __forceinline__ bool fe_is_zero(const Fe<L>& a) {
  uint32_t o = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) o |= a.w[i];
  return o == 0;
}

// Multiply by a small signed integer c by double-and-add (|c| < 2^31). The result equals
// the Montgomery product with the Montgomery image of c; an addition chain is cheaper
// than a product for the small coefficients constraint expressions carry.
template <int L>
__device__ __forceinline__ Fe<L> fe_mul_small(const Fe<L>& a, int32_t c, const FieldParams<L>& F) {
  uint32_t m = c < 0 ? static_cast<uint32_t>(-static_cast<int64_t>(c)) : static_cast<uint32_t>(c);
  Fe<L> acc = fe_zero<L>();
  Fe<L> base = a;
  bool first = true;
  while (m) {
    if (m & 1u) {
      acc = first ? base : fe_add(acc, base, F);
      first = false;
    }
    m >>= 1;
    if (m) base = fe_add(base, base, F);
  }
  if (c < 0) acc = fe_sub(fe_zero<L>(), acc, F);
  return acc;
}

template <int L>
__device__ __forceinline__ Fe<L> fe_shfl_down(const Fe<L>& a, int delta) {
  Fe<L> r;
#pragma unroll
  for (int i = 0; i < L; ++i) r.w[i] = __shfl_down_sync(0xffffffffu, a.w[i], delta);
  return r;
}

template <int L>
__device__ __forceinline__ Fe<L> fe_shfl(const Fe<L>& a, int src) {
  Fe<L> r;
#pragma unroll
  for (int i = 0; i < L; ++i) r.w[i] = __shfl_sync(0xffffffffu, a.w[i], src);
  return r;
}

}  // namespace sc
