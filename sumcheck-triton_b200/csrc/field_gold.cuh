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

}  // namespace sc

