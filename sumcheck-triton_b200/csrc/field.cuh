// Field elements and their arithmetic on the device.
//
// An element of a field with L 32-bit limbs is Fe<L>: little-endian limbs, Montgomery form
// (x R mod p, R = 2^(32 L)), always fully reduced (< p). Fully reduced Montgomery limbs are
// unique, so they are what the transcript hashes and the checksum sums, exactly as in the
// reference (cuda/src/field_sumcheck.cu:1046-1049, :857-907).
//
// Which Montgomery product runs is chosen per limb count by measurement on B200 (a probe of
// chained products per thread, 148 x 8 blocks; G products/s):
//
//   L = 1  inline-PTX mad.lo.cc / madc.hi.cc chain (field_ptx.cuh)     2.30  (C++ form 1.68)
//   L = 2  Goldilocks modulus: the special reduction below              0.81
//          any other modulus: CIOS with 64-bit intermediates (C++)     0.56  (PTX chains 0.51)
//   L = 4  CIOS with 64-bit intermediates                               0.167 (PTX chains 0.157)
//   L = 8  p < 2^255: even/odd-chain PTX product (ptx_mont_mul_eo)      0.065 (128 threads x 8 blocks/SM)
//          other moduli: CIOS with 64-bit intermediates                0.0456 (two-chain PTX 0.034)
//
// The even/odd form keeps the products of even and odd limbs in two accumulators, so each is
// one carry chain of fused multiply-adds: ncu counts 188 instructions a product, 136 of them
// on the FMA pipe and 52 on the ALU, against 458 (230 FMA, 221 ALU) for the C++ CIOS. From 4
// limbs up it is used whenever p < 2^(32 L - 1) (SC_MUL_EO; the BLS12-381 scalar field).
//
// All forms compute the same function: a b R^-1 mod p, fully reduced, for a, b < p. Modular
// add and subtract are inline-PTX add.cc/addc and sub.cc/subc chains for every L.
#pragma once
#include <cstdint>

#include "field_gold.cuh"
#include "field_ptx.cuh"

namespace sc {

constexpr int kMaxLimbs = 8;
constexpr int kMaxPoints = 8;  // t = 0..7, degree <= 7

// kFieldGoldilocksFma is the Goldilocks field with every carry on the FMA pipe (add and
// subtract too, field_gold.cuh): the compile-time shape kernels evaluate with it (process_pairs).
enum FieldKind : int { kFieldGeneric = 0, kFieldGoldilocks = 1, kFieldMersenne127 = 2, kFieldGoldilocksFma = 3 };

template <int L>
struct Fe {
  uint32_t w[L];
};

// The two constants every product needs. Passed by value as a kernel parameter, so it
// lives in the constant bank. KIND selects a special reduction for a known modulus.
template <int L, int KIND = kFieldGeneric>
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

// Goldilocks operations whose carries run on the FMA pipe (field_gold.cuh), by bit:
// 1 the product, 2 addition, 4 subtraction. Measured on B200 (plain_goldilocks, n = 24; the
// mixed stream's 64-bit group alone): ALU forms 1.94 ms / 6.14 ms; product on the FMA pipe
// 1.71 / 6.05; product, add and subtract 1.66 / 6.35 (the generic batched evaluator, whose
// adds are mostly point steps, lost). So the product runs on the FMA pipe everywhere and the
// compile-time shape kernels, alone, also add and subtract there (kFieldGoldilocksFma).
#ifndef SC_GOLD_FMA
#define SC_GOLD_FMA 1
#endif
#ifndef SC_GOLD_SHAPE_FMA
#define SC_GOLD_SHAPE_FMA 1
#endif


// The FMA-pipe Goldilocks forms need 1, 0 and 2^32 - 1 as values the compiler cannot fold:
// the modulus words p = (1, 2^32 - 1) of the kernel parameters.
template <int L, int K>
__device__ __forceinline__ GoldK gold_k(const FieldParams<L, K>& F) {
  return GoldK{F.p[0], F.p[0] >> 1, F.p[L - 1]};
}

template <int L, int K>
__device__ __forceinline__ Fe<L> fe_add(const Fe<L>& a, const Fe<L>& b, const FieldParams<L, K>& F) {
  Fe<L> r;
  if constexpr (L == 2 && (K == kFieldGoldilocksFma || (K == kFieldGoldilocks && (SC_GOLD_FMA & 2)))) {
    gold_add_fma(r.w, a.w, b.w, gold_k(F));
  } else {
    ptx_add_mod<L>(r.w, a.w, b.w, F.p);
  }
  return r;
}

template <int L, int K>
__device__ __forceinline__ Fe<L> fe_sub(const Fe<L>& a, const Fe<L>& b, const FieldParams<L, K>& F) {
  Fe<L> r;
  if constexpr (L == 2 && (K == kFieldGoldilocksFma || (K == kFieldGoldilocks && (SC_GOLD_FMA & 4)))) {
    gold_sub_fma(r.w, a.w, b.w, gold_k(F));
  } else {
    ptx_sub_mod<L>(r.w, a.w, b.w, F.p);
  }
  return r;
}

// CIOS (Koc-Acar-Kaliski 1996) with 64-bit intermediates and a fully carried L+2-word
// accumulator; the compiler chooses the multiply-add instructions.
template <int L>
__device__ __forceinline__ void cios_mul(uint32_t (&r)[L], const uint32_t (&a)[L], const uint32_t (&b)[L],
                                         const uint32_t (&p)[L], uint32_t np) {
  uint32_t t[L + 2];
#pragma unroll
  for (int i = 0; i < L + 2; ++i) t[i] = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    uint64_t c = 0;
#pragma unroll
    for (int j = 0; j < L; ++j) {
      const uint64_t uv = static_cast<uint64_t>(a[j]) * b[i] + t[j] + c;
      t[j] = static_cast<uint32_t>(uv);
      c = uv >> 32;
    }
    uint64_t s = static_cast<uint64_t>(t[L]) + c;
    t[L] = static_cast<uint32_t>(s);
    t[L + 1] = static_cast<uint32_t>(s >> 32);
    const uint32_t m = t[0] * np;
    c = (static_cast<uint64_t>(m) * p[0] + t[0]) >> 32;
#pragma unroll
    for (int j = 1; j < L; ++j) {
      const uint64_t uv = static_cast<uint64_t>(m) * p[j] + t[j] + c;
      t[j - 1] = static_cast<uint32_t>(uv);
      c = uv >> 32;
    }
    s = static_cast<uint64_t>(t[L]) + c;
    t[L - 1] = static_cast<uint32_t>(s);
    t[L] = t[L + 1] + static_cast<uint32_t>(s >> 32);
    t[L + 1] = 0;
  }
  uint32_t d[L];
  uint64_t br = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    const uint64_t x = static_cast<uint64_t>(t[i]) - p[i] - br;
    d[i] = static_cast<uint32_t>(x);
    br = (x >> 63) & 1;
  }
  const bool below = (t[L] == 0) && br;  // t < p: keep t
#pragma unroll
  for (int i = 0; i < L; ++i) r[i] = below ? t[i] : d[i];
}

// Montgomery product for p = 2^64 - 2^32 + 1 and R = 2^64 (x, y < p):
// with x y = h 2^64 + l, -p^-1 = -(1 + 2^32) mod 2^64, so a = l (1 + 2^32) mod 2^64 (carry
// e out of the 32-bit halves) satisfies x y - a p = 0 mod 2^64, and
// (x y - a p) / 2^64 = h - b with b = a - (a >> 32) - e, 0 <= b < p; one conditional
// addition of p makes h - b fully reduced. (Derivation in the comment of gold_mul's test.)
__device__ __forceinline__ void gold_mul(uint32_t (&r)[2], const uint32_t (&x32)[2], const uint32_t (&y32)[2]) {
  const uint64_t x = (static_cast<uint64_t>(x32[1]) << 32) | x32[0];
  const uint64_t y = (static_cast<uint64_t>(y32[1]) << 32) | y32[0];
  const uint64_t l = x * y;
  const uint64_t h = __umul64hi(x, y);
  const uint64_t a = l + (l << 32);
  const uint64_t e = a < l ? 1u : 0u;
  const uint64_t b = a - (a >> 32) - e;
  uint64_t res = h - b;
  if (h < b) res += 0xFFFFFFFF00000001ull;
  r[0] = static_cast<uint32_t>(res);
  r[1] = static_cast<uint32_t>(res >> 32);
}

#ifndef SC_OUTLINE_MIN_LIMBS
#define SC_OUTLINE_MIN_LIMBS 4
#endif

// An 8-limb product is ~500 instructions; kernels that inline dozens of them outgrow the
// instruction cache (measured on B200: the 8-limb round kernels stalled on instruction fetch
// first; out of line, the 256-bit proofs ran 20-25% faster, the 4-limb served stream ~3%).
// From SC_OUTLINE_MIN_LIMBS limbs up the product is one out-of-line function, operands and
// result passed by value in registers.
#ifndef SC_MUL_EO
#define SC_MUL_EO 1
#endif
// Moduli whose low words are p_0 = 1, p_1 = 2^32 - 1 (the BLS12-381 scalar field) use the
// even/odd form with those words' multiplies done on the ALU (ptx_mont_mul_eo1): the product
// is bound by the FMA-heavy pipe (ncu on a probe of chained products: 82% busy at 3 and at 8
// blocks/SM, 55 G products/s either way), so fewer multiplies is what makes it faster.
#ifndef SC_MUL_EO1
#define SC_MUL_EO1 1
#endif
// The Montgomery product of a generic modulus: the even/odd-chain form when it applies
// (p < 2^(32L - 1), from 4 limbs up), else CIOS with 64-bit intermediates.
template <int L>
__device__ __forceinline__ void mont_mul_generic(uint32_t (&r)[L], const uint32_t (&a)[L], const uint32_t (&b)[L],
                                                 const FieldParams<L, kFieldGeneric>& F) {
#if SC_MUL_EO
  if constexpr (L >= 4) {
    if (F.p[L - 1] < 0x80000000u) {
#if SC_MUL_EO1
      if (F.p[0] == 1u && F.p[1] == 0xFFFFFFFFu) {
        ptx_mont_mul_eo1<L>(r, a, b, F.p, F.np);
        return;
      }
#endif
      ptx_mont_mul_eo<L>(r, a, b, F.p, F.np);
      return;
    }
  }
#endif
  cios_mul<L>(r, a, b, F.p, F.np);
}

template <int L>
__device__ __noinline__ Fe<L> cios_mul_call(const Fe<L> a, const Fe<L> b, const FieldParams<L, kFieldGeneric> F) {
  Fe<L> r;
  mont_mul_generic<L>(r.w, a.w, b.w, F);
  return r;
}

// Montgomery product for p = 2^127 - 1 and R = 2^128 (x, y < p): R = 2 (mod p), so
// x y R^-1 = (x y mod p) 2^126, and multiplying a 127-bit residue by 2^126 = 2^-1 is a
// rotation right by one bit. x y < 2^254 = h 2^127 + l reduces to h + l < 2^128, then
// (s mod 2^127) + (s >> 127) <= p, then one conditional subtraction of p.
__device__ __forceinline__ void m127_mul(uint32_t (&r)[4], const uint32_t (&x)[4], const uint32_t (&y)[4]) {
  uint32_t t[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) t[i] = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    uint64_t c = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint64_t uv = static_cast<uint64_t>(x[j]) * y[i] + t[i + j] + c;
      t[i + j] = static_cast<uint32_t>(uv);
      c = uv >> 32;
    }
    t[i + 4] = static_cast<uint32_t>(c);
  }
  // l = t mod 2^127, h = t >> 127 (both < 2^127); s = l + h
  uint32_t h[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) h[i] = (t[i + 3] >> 31) | (t[i + 4] << 1);
  t[3] &= 0x7fffffffu;
  uint32_t sw[4];
  uint64_t c = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint64_t v = static_cast<uint64_t>(t[i]) + h[i] + c;
    sw[i] = static_cast<uint32_t>(v);
    c = v >> 32;
  }
  // s < 2^128: fold bit 127 back in (2^127 = 1)
  const uint32_t top = sw[3] >> 31;
  sw[3] &= 0x7fffffffu;
  c = top;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint64_t v = static_cast<uint64_t>(sw[i]) + c;
    sw[i] = static_cast<uint32_t>(v);
    c = v >> 32;
  }
  // now s <= p; s == p means 0
  const bool is_p = sw[0] == 0xffffffffu && sw[1] == 0xffffffffu && sw[2] == 0xffffffffu && sw[3] == 0x7fffffffu;
  if (is_p) sw[0] = sw[1] = sw[2] = sw[3] = 0;
  // times 2^126 = 2^-1: rotate the 127-bit value right by one
  const uint32_t low = sw[0] & 1u;
  r[0] = (sw[0] >> 1) | (sw[1] << 31);
  r[1] = (sw[1] >> 1) | (sw[2] << 31);
  r[2] = (sw[2] >> 1) | (sw[3] << 31);
  r[3] = (sw[3] >> 1) | (low << 30);
}

static __device__ __noinline__ Fe<4> m127_mul_call(const Fe<4> a, const Fe<4> b) {
  Fe<4> r;
  m127_mul(r.w, a.w, b.w);
  return r;
}

template <int L, int K>
__device__ __forceinline__ Fe<L> fe_mul(const Fe<L>& a, const Fe<L>& b, const FieldParams<L, K>& F) {
  Fe<L> r;
  if constexpr (L == 2 && (K == kFieldGoldilocksFma || (K == kFieldGoldilocks && (SC_GOLD_FMA & 1)))) {
    gold_mul_fma(r.w, a.w, b.w, gold_k(F));
  } else if constexpr (K == kFieldGoldilocks && L == 2) {
    gold_mul(r.w, a.w, b.w);
  } else if constexpr (K == kFieldMersenne127 && L == 4) {
    r = m127_mul_call(a, b);
  } else if constexpr (L == 1) {
    ptx_mont_mul<1>(r.w, a.w, b.w, F.p, F.np);
  } else if constexpr (L >= SC_OUTLINE_MIN_LIMBS && K == kFieldGeneric) {
    r = cios_mul_call<L>(a, b, F);
  } else if constexpr (K == kFieldGeneric) {
    mont_mul_generic<L>(r.w, a.w, b.w, F);
  } else {
    cios_mul<L>(r.w, a.w, b.w, F.p, F.np);
  }
  return r;
}

// Lazy Goldilocks arithmetic (field_gold.cuh): values are any representative in [0, 2^64)
// between operations and are made canonical (gold_canon) only where they leave a thread.
// Which forms, measured on B200 (plain_goldilocks n = 24 p50 / the mixed stream's 64-bit
// group alone, 240 proofs; canonical arithmetic 1.65 / 6.07 ms):
//   point steps (value + canonical difference) on the ALU, SC_GOLD_LAZY_STEP_ALU = 1:
//     1.60 / 5.93 ms; the same on the FMA pipe (five multiply-adds): 1.64 / 6.10 ms;
//   the product gold_mul_fma (exact on any operands), SC_GOLD_MUL_ANY = 0; gold_mul_any, with
//     four more of its steps on the FMA pipe, took the shape kernel to 1.72 ms.
__device__ __forceinline__ Fe<2> gl_add(const Fe<2>& a, const Fe<2>& b, const GoldK k) {
  Fe<2> r;
  gold_add_lazy(r.w, a.w, b.w, k);
  return r;
}
#ifndef SC_GOLD_LAZY_STEP_ALU
#define SC_GOLD_LAZY_STEP_ALU 1
#endif
#ifndef SC_GOLD_MUL_ANY
#define SC_GOLD_MUL_ANY 0
#endif
__device__ __forceinline__ Fe<2> gl_add_c(const Fe<2>& a, const Fe<2>& b_canonical, const GoldK k) {
  Fe<2> r;
#if SC_GOLD_LAZY_STEP_ALU
  gold_add_lazy_c_alu(r.w, a.w, b_canonical.w, k);
#else
  gold_add_lazy_c(r.w, a.w, b_canonical.w, k);
#endif
  return r;
}
__device__ __forceinline__ Fe<2> gl_sub(const Fe<2>& a, const Fe<2>& b, const GoldK k) {
  Fe<2> r;
  gold_sub_lazy(r.w, a.w, b.w, k);
  return r;
}
__device__ __forceinline__ Fe<2> gl_mul(const Fe<2>& a, const Fe<2>& b, const GoldK k) {
  Fe<2> r;
#if SC_GOLD_MUL_ANY
  gold_mul_any(r.w, a.w, b.w, k);
#else
  gold_mul_fma(r.w, a.w, b.w, k);  // also exact on operands in [0, 2^64) (see gold_mul_any)
#endif
  return r;
}
__device__ __forceinline__ Fe<2> gl_canon(const Fe<2>& a, const GoldK k) {
  Fe<2> r;
  gold_canon(r.w, a.w, k);
  return r;
}

template <int L>
__device__ __forceinline__ bool fe_is_zero(const Fe<L>& a) {
  uint32_t o = 0;
#pragma unroll
  for (int i = 0; i < L; ++i) o |= a.w[i];
  return o == 0;
}

// Multiply by a small non-negative integer c by double-and-add. The result equals the
// Montgomery product with c's Montgomery image; an addition chain is cheaper than a product
// for the small coefficients constraint expressions carry.
template <int L, int K>
__device__ __forceinline__ Fe<L> fe_mul_small(const Fe<L>& a, uint32_t m, const FieldParams<L, K>& F) {
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
