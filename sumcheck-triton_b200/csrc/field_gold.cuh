// Goldilocks (p = 2^64 - 2^32 + 1, R = 2^64) arithmetic whose carries run on the FMA pipe.
//
// The 2-limb kernels are bound by the ALU pipe, which executes the add-with-carry,
// compare and select instructions of 64-bit modular arithmetic on 32-bit words, while the
// FMA pipe, which executes multiply-adds, idles (ncu on the zerocheck round kernel: ALU
// 64-72% of peak, FMA 11%). A carry chain of multiply-adds (mad.lo.cc / madc) runs on the
// FMA pipe, carries included, so these forms move work across: a + b is formed as
// a * one + b, the borrow mask of a subtraction becomes a multiplier of p.
//
// `one`, `zero` and `eps` (= 2^32 - 1) must be values the compiler cannot see (the field's
// own modulus words from the kernel parameters: p = (1, 2^32 - 1)), or it would fold the
// multiplies back into ALU additions. Canonical inputs (< p), canonical outputs; each
// statement is one asm block (the carry flag does not survive between statements).
// Checked against big-integer arithmetic by tests/test_field_ptx_emulated.py.
#pragma once
#include <cstdint>

namespace sc {

struct GoldK {
  uint32_t one, zero, eps;
};

// r = a + b mod p: s = a + b; t = s + (2^64 - p); t if either carried, else s.
__device__ __forceinline__ void gold_add_fma(uint32_t (&r)[2], const uint32_t (&a)[2], const uint32_t (&b)[2],
                                             const GoldK k) {
  asm("{\n\t.reg .u32 s0, s1, t0, t1, c;\n\t.reg .pred q;\n\t"
      "mad.lo.cc.u32 s0, %2, %6, %4;\n\t"
      "madc.lo.cc.u32 s1, %3, %6, %5;\n\t"
      "madc.lo.u32 c, %7, %7, %7;\n\t"
      "mad.lo.cc.u32 t0, s0, %6, %8;\n\t"
      "madc.lo.cc.u32 t1, s1, %6, %7;\n\t"
      "madc.lo.u32 c, %7, %7, c;\n\t"
      "setp.ne.u32 q, c, 0;\n\t"
      "selp.b32 %0, t0, s0, q;\n\t"
      "selp.b32 %1, t1, s1, q;\n\t}"
      : "=&r"(r[0]), "=&r"(r[1])
      : "r"(a[0]), "r"(a[1]), "r"(b[0]), "r"(b[1]), "r"(k.one), "r"(k.zero), "r"(k.eps));
}

// r = a - b mod p: d = a - b; m = -borrow (0 or 2^32 - 1, from the subtraction's own flag);
// then d + p when m is set, as multiply-adds: m m = 1 (mod 2^32) into the low word and m into
// the high word, p being (1, 2^32 - 1). (A subtraction's flag is read by subc only: an add or
// multiply-add reading it is not portable, and gave wrong results when compiled.)
__device__ __forceinline__ void gold_sub_fma(uint32_t (&r)[2], const uint32_t (&a)[2], const uint32_t (&b)[2],
                                             const GoldK k) {
  asm("{\n\t.reg .u32 d0, d1, m;\n\t"
      "sub.cc.u32 d0, %2, %4;\n\t"
      "subc.cc.u32 d1, %3, %5;\n\t"
      "subc.u32 m, %7, %7;\n\t"
      "mad.lo.cc.u32 %0, m, m, d0;\n\t"
      "madc.lo.u32 %1, m, %6, d1;\n\t}"
      : "=&r"(r[0]), "=&r"(r[1])
      : "r"(a[0]), "r"(a[1]), "r"(b[0]), "r"(b[1]), "r"(k.one), "r"(k.zero), "r"(k.eps));
}

// Montgomery product x y R^-1 mod p (the reduction of gold_mul in field.cuh): the 128-bit
// product t on multiply-add chains; a = l (1 + 2^32) mod 2^64 with carry e; b = a - (a >> 32)
// - e; r = h - b, plus p on a borrow (added as in gold_sub_fma).
__device__ __forceinline__ void gold_mul_fma(uint32_t (&r)[2], const uint32_t (&x)[2], const uint32_t (&y)[2],
                                             const GoldK k) {
  asm("{\n\t.reg .u32 t0, t1, t2, t3, a1, e, b0, b1, r0, r1, m;\n\t"
      "mul.lo.u32 t0, %2, %4;\n\t"
      "mul.hi.u32 t1, %2, %4;\n\t"
      "mul.lo.u32 t2, %3, %5;\n\t"
      "mul.hi.u32 t3, %3, %5;\n\t"
      "mad.lo.cc.u32 t1, %2, %5, t1;\n\t"
      "madc.hi.cc.u32 t2, %2, %5, t2;\n\t"
      "madc.lo.u32 t3, %7, %7, t3;\n\t"
      "mad.lo.cc.u32 t1, %3, %4, t1;\n\t"
      "madc.hi.cc.u32 t2, %3, %4, t2;\n\t"
      "madc.lo.u32 t3, %7, %7, t3;\n\t"
      "mad.lo.cc.u32 a1, t0, %6, t1;\n\t"
      "madc.lo.u32 e, %7, %7, %7;\n\t"
      "sub.cc.u32 b0, t0, a1;\n\t"
      "subc.u32 b1, a1, 0;\n\t"
      "sub.cc.u32 b0, b0, e;\n\t"
      "subc.u32 b1, b1, 0;\n\t"
      "sub.cc.u32 r0, t2, b0;\n\t"
      "subc.cc.u32 r1, t3, b1;\n\t"
      "subc.u32 m, %7, %7;\n\t"
      "mad.lo.cc.u32 %0, m, m, r0;\n\t"
      "madc.lo.u32 %1, m, %6, r1;\n\t}"
      : "=&r"(r[0]), "=&r"(r[1])
      : "r"(x[0]), "r"(x[1]), "r"(y[0]), "r"(y[1]), "r"(k.one), "r"(k.zero), "r"(k.eps));
}

// Lazy forms: operands anywhere in [0, 2^64) (any representative of their residue), results
// in [0, 2^64), nothing canonical until gold_canon. 2^64 = 2^32 - 1 = eps (mod p), so a carry
// out of bit 63 is worth eps and a borrow -eps.

// r = a + b for a in [0, 2^64) and b < p: s = a + b, then s + eps on a carry, which cannot
// carry again (a + b - 2^64 + eps <= p - 2 + eps < 2^64). Five multiply-adds.
__device__ __forceinline__ void gold_add_lazy_c(uint32_t (&r)[2], const uint32_t (&a)[2], const uint32_t (&b)[2],
                                                const GoldK k) {
  asm("{\n\t.reg .u32 s0, s1, c;\n\t"
      "mad.lo.cc.u32 s0, %2, %6, %4;\n\t"
      "madc.lo.cc.u32 s1, %3, %6, %5;\n\t"
      "madc.lo.u32 c, %7, %7, %7;\n\t"
      "mad.lo.cc.u32 %0, c, %8, s0;\n\t"
      "madc.lo.u32 %1, %7, %7, s1;\n\t}"
      : "=&r"(r[0]), "=&r"(r[1])
      : "r"(a[0]), "r"(a[1]), "r"(b[0]), "r"(b[1]), "r"(k.one), "r"(k.zero), "r"(k.eps));
}

// gold_add_lazy_c on the ALU pipe: the carry c becomes the mask -c (0 or 2^32 - 1 = eps).
__device__ __forceinline__ void gold_add_lazy_c_alu(uint32_t (&r)[2], const uint32_t (&a)[2], const uint32_t (&b)[2],
                                                    const GoldK k) {
  asm("{\n\t.reg .u32 s0, s1, c, m;\n\t"
      "add.cc.u32 s0, %2, %4;\n\t"
      "addc.cc.u32 s1, %3, %5;\n\t"
      "addc.u32 c, %7, %7;\n\t"
      "sub.u32 m, %7, c;\n\t"
      "add.cc.u32 %0, s0, m;\n\t"
      "addc.u32 %1, s1, %7;\n\t}"
      : "=&r"(r[0]), "=&r"(r[1])
      : "r"(a[0]), "r"(a[1]), "r"(b[0]), "r"(b[1]), "r"(k.one), "r"(k.zero), "r"(k.eps));
}

// r = a + b for a, b in [0, 2^64): the carry's eps is added, and once more if that carried
// (then the sum is below 2 eps and a third carry is impossible). Eight multiply-adds.
__device__ __forceinline__ void gold_add_lazy(uint32_t (&r)[2], const uint32_t (&a)[2], const uint32_t (&b)[2],
                                              const GoldK k) {
  asm("{\n\t.reg .u32 s0, s1, t0, t1, c;\n\t"
      "mad.lo.cc.u32 s0, %2, %6, %4;\n\t"
      "madc.lo.cc.u32 s1, %3, %6, %5;\n\t"
      "madc.lo.u32 c, %7, %7, %7;\n\t"
      "mad.lo.cc.u32 t0, c, %8, s0;\n\t"
      "madc.lo.cc.u32 t1, %7, %7, s1;\n\t"
      "madc.lo.u32 c, %7, %7, %7;\n\t"
      "mad.lo.cc.u32 %0, c, %8, t0;\n\t"
      "madc.lo.u32 %1, %7, %7, t1;\n\t}"
      : "=&r"(r[0]), "=&r"(r[1])
      : "r"(a[0]), "r"(a[1]), "r"(b[0]), "r"(b[1]), "r"(k.one), "r"(k.zero), "r"(k.eps));
}

// r = a - b for a, b in [0, 2^64): d = a - b mod 2^64; on a borrow the value is d - 2^64 = d -
// eps (mod p), formed as d + p (mod 2^64) under the mask m; that addition fails to carry
// exactly when d < eps, and then p is added once more (mask f = m + carry: all ones only for a
// borrow without the carry), giving d + 2p - 2^64 < 2^64.
__device__ __forceinline__ void gold_sub_lazy(uint32_t (&r)[2], const uint32_t (&a)[2], const uint32_t (&b)[2],
                                              const GoldK k) {
  asm("{\n\t.reg .u32 d0, d1, x0, x1, m, f;\n\t"
      "sub.cc.u32 d0, %2, %4;\n\t"
      "subc.cc.u32 d1, %3, %5;\n\t"
      "subc.u32 m, %7, %7;\n\t"
      "mad.lo.cc.u32 x0, m, m, d0;\n\t"
      "madc.lo.cc.u32 x1, m, %6, d1;\n\t"
      "madc.lo.u32 f, m, %6, %7;\n\t"
      "mad.lo.cc.u32 %0, f, f, x0;\n\t"
      "madc.lo.u32 %1, f, %6, x1;\n\t}"
      : "=&r"(r[0]), "=&r"(r[1])
      : "r"(a[0]), "r"(a[1]), "r"(b[0]), "r"(b[1]), "r"(k.one), "r"(k.zero), "r"(k.eps));
}

// The canonical representative of a in [0, 2^64): a >= p exactly when a + eps carries, and
// then a - p = a + eps - 2^64.
__device__ __forceinline__ void gold_canon(uint32_t (&r)[2], const uint32_t (&a)[2], const GoldK k) {
  asm("{\n\t.reg .u32 t0, t1, c;\n\t"
      "mad.lo.cc.u32 t0, %2, %4, %6;\n\t"
      "madc.lo.cc.u32 t1, %3, %4, %5;\n\t"
      "madc.lo.u32 c, %5, %5, %5;\n\t"
      "mad.lo.cc.u32 %0, c, %6, %2;\n\t"
      "madc.lo.u32 %1, %5, %5, %3;\n\t}"
      : "=&r"(r[0]), "=&r"(r[1])
      : "r"(a[0]), "r"(a[1]), "r"(k.one), "r"(k.zero), "r"(k.eps));
}

// The Montgomery product of gold_mul_fma with b = a - (a >> 32) - e also on multiply-adds:
// a - (a >> 32) = a0 + a1 (2^32 - 1) = a0 + a1 eps exactly, and - e is + e (2^64 - 1), whose
// words are (eps, eps). Operands in [0, 2^64): t < 2^128 keeps (t - a p) / 2^64 in (-p, 2^64),
// so h - b, plus p on a borrow, lies in [0, 2^64) (below p when both operands are below p).
__device__ __forceinline__ void gold_mul_any(uint32_t (&r)[2], const uint32_t (&x)[2], const uint32_t (&y)[2],
                                             const GoldK k) {
  asm("{\n\t.reg .u32 t0, t1, t2, t3, a1, e, b0, b1, r0, r1, m;\n\t"
      "mul.lo.u32 t0, %2, %4;\n\t"
      "mul.hi.u32 t1, %2, %4;\n\t"
      "mul.lo.u32 t2, %3, %5;\n\t"
      "mul.hi.u32 t3, %3, %5;\n\t"
      "mad.lo.cc.u32 t1, %2, %5, t1;\n\t"
      "madc.hi.cc.u32 t2, %2, %5, t2;\n\t"
      "madc.lo.u32 t3, %7, %7, t3;\n\t"
      "mad.lo.cc.u32 t1, %3, %4, t1;\n\t"
      "madc.hi.cc.u32 t2, %3, %4, t2;\n\t"
      "madc.lo.u32 t3, %7, %7, t3;\n\t"
      "mad.lo.cc.u32 a1, t0, %6, t1;\n\t"
      "madc.lo.u32 e, %7, %7, %7;\n\t"
      "mad.lo.cc.u32 b0, a1, %8, t0;\n\t"
      "madc.hi.u32 b1, a1, %8, %7;\n\t"
      "mad.lo.cc.u32 b0, e, %8, b0;\n\t"
      "madc.lo.u32 b1, e, %8, b1;\n\t"
      "sub.cc.u32 r0, t2, b0;\n\t"
      "subc.cc.u32 r1, t3, b1;\n\t"
      "subc.u32 m, %7, %7;\n\t"
      "mad.lo.cc.u32 %0, m, m, r0;\n\t"
      "madc.lo.u32 %1, m, %6, r1;\n\t}"
      : "=&r"(r[0]), "=&r"(r[1])
      : "r"(x[0]), "r"(x[1]), "r"(y[0]), "r"(y[1]), "r"(k.one), "r"(k.zero), "r"(k.eps));
}

}  // namespace sc
