// GENERATED by gen_field_ptx.py -- do not edit by hand.
// Inline-PTX carry chains of the field arithmetic for L = 1, 2, 4, 8 limbs.
#pragma once
#include <cstdint>

template <int L> __device__ __forceinline__ void ptx_mont_mul(uint32_t (&r)[L], const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L], uint32_t np);
template <int L> __device__ __forceinline__ void ptx_add_mod(uint32_t (&r)[L], const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L]);
template <int L> __device__ __forceinline__ void ptx_sub_mod(uint32_t (&r)[L], const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L]);

// ---------------- L = 1 ----------------
template <> __device__ __forceinline__ void ptx_mont_mul<1>(uint32_t (&r)[1], const uint32_t (&a)[1], const uint32_t (&b)[1], const uint32_t (&p)[1], uint32_t np) {
    uint32_t hi, c;
    asm(
        "{\n\t"
        ".reg .u32 lo, m;\n\t"
        "mul.lo.u32 lo, %2, %3;\n\t"
        "mul.hi.u32 %0, %2, %3;\n\t"
        "mul.lo.u32 m, lo, %5;\n\t"
        "mad.lo.cc.u32 lo, m, %4, lo;\n\t"
        "madc.hi.cc.u32 %0, m, %4, %0;\n\t"
        "addc.u32 %1, 0, 0;\n\t"
        "}"
        : "=&r"(hi), "=&r"(c)
        : "r"(a[0]), "r"(b[0]), "r"(p[0]), "r"(np));
    uint32_t d, bw;
    asm(
        "sub.cc.u32 %0, %2, %4;\n\t"
        "subc.u32 %1, %3, 0;"
        : "=&r"(d), "=&r"(bw)
        : "r"(hi), "r"(c), "r"(p[0]));
    r[0] = bw ? hi : d;
}

template <> __device__ __forceinline__ void ptx_add_mod<1>(uint32_t (&r)[1], const uint32_t (&a)[1], const uint32_t (&b)[1], const uint32_t (&p)[1]) {
    uint32_t s[1], d[1], c, bw;
    asm(
        "add.cc.u32 %0, %2, %3;\n\t"
        "addc.u32 %1, 0, 0;"
        : "=&r"(s[0]), "=&r"(c)
        : "r"(a[0]), "r"(b[0]));
    asm(
        "sub.cc.u32 %0, %2, %4;\n\t"
        "subc.u32 %1, %3, 0;"
        : "=&r"(d[0]), "=&r"(bw)
        : "r"(s[0]), "r"(c), "r"(p[0]));
#pragma unroll
    for (int j = 0; j < 1; ++j) r[j] = bw ? s[j] : d[j];
}

template <> __device__ __forceinline__ void ptx_sub_mod<1>(uint32_t (&r)[1], const uint32_t (&a)[1], const uint32_t (&b)[1], const uint32_t (&p)[1]) {
    uint32_t d[1], mask, q[1];
    asm(
        "sub.cc.u32 %0, %2, %3;\n\t"
        "subc.u32 %1, 0, 0;"
        : "=&r"(d[0]), "=&r"(mask)
        : "r"(a[0]), "r"(b[0]));
#pragma unroll
    for (int j = 0; j < 1; ++j) q[j] = p[j] & mask;
    asm(
        "add.u32 %0, %1, %2;"
        : "=&r"(r[0])
        : "r"(d[0]), "r"(q[0]));
}

// ---------------- L = 2 ----------------
template <> __device__ __forceinline__ void ptx_mont_mul<2>(uint32_t (&r)[2], const uint32_t (&a)[2], const uint32_t (&b)[2], const uint32_t (&p)[2], uint32_t np) {
    uint32_t t[4];
    asm(
        "mul.lo.u32 %0, %3, %5;\n\t"
        "mul.lo.u32 %1, %4, %5;\n\t"
        "mov.u32 %2, 0;"
        : "=&r"(t[0]), "=&r"(t[1]), "=&r"(t[2])
        : "r"(a[0]), "r"(a[1]), "r"(b[0]));
    asm(
        "mad.hi.cc.u32 %1, %3, %5, %1;\n\t"
        "madc.hi.u32 %2, %4, %5, %2;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2])
        : "r"(a[0]), "r"(a[1]), "r"(b[0]));
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      if (i > 0) {
      asm(
          "mad.lo.cc.u32 %0, %3, %5, %0;\n\t"
          "madc.lo.cc.u32 %1, %4, %5, %1;\n\t"
          "addc.u32 %2, %2, 0;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2])
          : "r"(a[0]), "r"(a[1]), "r"(b[i]));
      asm(
          "mad.hi.cc.u32 %1, %3, %5, %1;\n\t"
          "madc.hi.u32 %2, %4, %5, %2;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2])
          : "r"(a[0]), "r"(a[1]), "r"(b[i]));
      }
      const uint32_t m = t[0] * np;
      asm(
          "mad.lo.cc.u32 %0, %6, %4, %0;\n\t"
          "madc.lo.cc.u32 %1, %6, %5, %1;\n\t"
          "addc.cc.u32 %2, %2, 0;\n\t"
          "addc.u32 %3, 0, 0;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "=&r"(t[3])
          : "r"(p[0]), "r"(p[1]), "r"(m));
      asm(
          "mad.hi.cc.u32 %1, %6, %4, %1;\n\t"
          "madc.hi.cc.u32 %2, %6, %5, %2;\n\t"
          "addc.u32 %3, %3, 0;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3])
          : "r"(p[0]), "r"(p[1]), "r"(m));
#pragma unroll
      for (int j = 0; j <= 2; ++j) t[j] = t[j + 1];
    }
    uint32_t d[2], bw;
    asm(
        "sub.cc.u32 %0, %3, %6;\n\t"
        "subc.cc.u32 %1, %4, %7;\n\t"
        "subc.u32 %2, %5, 0;"
        : "=&r"(d[0]), "=&r"(d[1]), "=&r"(bw)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(p[0]), "r"(p[1]));
#pragma unroll
    for (int j = 0; j < 2; ++j) r[j] = bw ? t[j] : d[j];
}

template <> __device__ __forceinline__ void ptx_add_mod<2>(uint32_t (&r)[2], const uint32_t (&a)[2], const uint32_t (&b)[2], const uint32_t (&p)[2]) {
    uint32_t s[2], d[2], c, bw;
    asm(
        "add.cc.u32 %0, %3, %5;\n\t"
        "addc.cc.u32 %1, %4, %6;\n\t"
        "addc.u32 %2, 0, 0;"
        : "=&r"(s[0]), "=&r"(s[1]), "=&r"(c)
        : "r"(a[0]), "r"(a[1]), "r"(b[0]), "r"(b[1]));
    asm(
        "sub.cc.u32 %0, %3, %6;\n\t"
        "subc.cc.u32 %1, %4, %7;\n\t"
        "subc.u32 %2, %5, 0;"
        : "=&r"(d[0]), "=&r"(d[1]), "=&r"(bw)
        : "r"(s[0]), "r"(s[1]), "r"(c), "r"(p[0]), "r"(p[1]));
#pragma unroll
    for (int j = 0; j < 2; ++j) r[j] = bw ? s[j] : d[j];
}

template <> __device__ __forceinline__ void ptx_sub_mod<2>(uint32_t (&r)[2], const uint32_t (&a)[2], const uint32_t (&b)[2], const uint32_t (&p)[2]) {
    uint32_t d[2], mask, q[2];
    asm(
        "sub.cc.u32 %0, %3, %5;\n\t"
        "subc.cc.u32 %1, %4, %6;\n\t"
        "subc.u32 %2, 0, 0;"
        : "=&r"(d[0]), "=&r"(d[1]), "=&r"(mask)
        : "r"(a[0]), "r"(a[1]), "r"(b[0]), "r"(b[1]));
#pragma unroll
    for (int j = 0; j < 2; ++j) q[j] = p[j] & mask;
    asm(
        "add.cc.u32 %0, %2, %4;\n\t"
        "addc.u32 %1, %3, %5;"
        : "=&r"(r[0]), "=&r"(r[1])
        : "r"(d[0]), "r"(d[1]), "r"(q[0]), "r"(q[1]));
}

// ---------------- L = 4 ----------------
template <> __device__ __forceinline__ void ptx_mont_mul<4>(uint32_t (&r)[4], const uint32_t (&a)[4], const uint32_t (&b)[4], const uint32_t (&p)[4], uint32_t np) {
    uint32_t t[6];
    asm(
        "mul.lo.u32 %0, %5, %9;\n\t"
        "mul.lo.u32 %1, %6, %9;\n\t"
        "mul.lo.u32 %2, %7, %9;\n\t"
        "mul.lo.u32 %3, %8, %9;\n\t"
        "mov.u32 %4, 0;"
        : "=&r"(t[0]), "=&r"(t[1]), "=&r"(t[2]), "=&r"(t[3]), "=&r"(t[4])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]));
    asm(
        "mad.hi.cc.u32 %1, %5, %9, %1;\n\t"
        "madc.hi.cc.u32 %2, %6, %9, %2;\n\t"
        "madc.hi.cc.u32 %3, %7, %9, %3;\n\t"
        "madc.hi.u32 %4, %8, %9, %4;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (i > 0) {
      asm(
          "mad.lo.cc.u32 %0, %5, %9, %0;\n\t"
          "madc.lo.cc.u32 %1, %6, %9, %1;\n\t"
          "madc.lo.cc.u32 %2, %7, %9, %2;\n\t"
          "madc.lo.cc.u32 %3, %8, %9, %3;\n\t"
          "addc.u32 %4, %4, 0;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4])
          : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[i]));
      asm(
          "mad.hi.cc.u32 %1, %5, %9, %1;\n\t"
          "madc.hi.cc.u32 %2, %6, %9, %2;\n\t"
          "madc.hi.cc.u32 %3, %7, %9, %3;\n\t"
          "madc.hi.u32 %4, %8, %9, %4;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4])
          : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[i]));
      }
      const uint32_t m = t[0] * np;
      asm(
          "mad.lo.cc.u32 %0, %10, %6, %0;\n\t"
          "madc.lo.cc.u32 %1, %10, %7, %1;\n\t"
          "madc.lo.cc.u32 %2, %10, %8, %2;\n\t"
          "madc.lo.cc.u32 %3, %10, %9, %3;\n\t"
          "addc.cc.u32 %4, %4, 0;\n\t"
          "addc.u32 %5, 0, 0;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "=&r"(t[5])
          : "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(m));
      asm(
          "mad.hi.cc.u32 %1, %10, %6, %1;\n\t"
          "madc.hi.cc.u32 %2, %10, %7, %2;\n\t"
          "madc.hi.cc.u32 %3, %10, %8, %3;\n\t"
          "madc.hi.cc.u32 %4, %10, %9, %4;\n\t"
          "addc.u32 %5, %5, 0;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5])
          : "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(m));
#pragma unroll
      for (int j = 0; j <= 4; ++j) t[j] = t[j + 1];
    }
    uint32_t d[4], bw;
    asm(
        "sub.cc.u32 %0, %5, %10;\n\t"
        "subc.cc.u32 %1, %6, %11;\n\t"
        "subc.cc.u32 %2, %7, %12;\n\t"
        "subc.cc.u32 %3, %8, %13;\n\t"
        "subc.u32 %4, %9, 0;"
        : "=&r"(d[0]), "=&r"(d[1]), "=&r"(d[2]), "=&r"(d[3]), "=&r"(bw)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]));
#pragma unroll
    for (int j = 0; j < 4; ++j) r[j] = bw ? t[j] : d[j];
}

template <> __device__ __forceinline__ void ptx_add_mod<4>(uint32_t (&r)[4], const uint32_t (&a)[4], const uint32_t (&b)[4], const uint32_t (&p)[4]) {
    uint32_t s[4], d[4], c, bw;
    asm(
        "add.cc.u32 %0, %5, %9;\n\t"
        "addc.cc.u32 %1, %6, %10;\n\t"
        "addc.cc.u32 %2, %7, %11;\n\t"
        "addc.cc.u32 %3, %8, %12;\n\t"
        "addc.u32 %4, 0, 0;"
        : "=&r"(s[0]), "=&r"(s[1]), "=&r"(s[2]), "=&r"(s[3]), "=&r"(c)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]));
    asm(
        "sub.cc.u32 %0, %5, %10;\n\t"
        "subc.cc.u32 %1, %6, %11;\n\t"
        "subc.cc.u32 %2, %7, %12;\n\t"
        "subc.cc.u32 %3, %8, %13;\n\t"
        "subc.u32 %4, %9, 0;"
        : "=&r"(d[0]), "=&r"(d[1]), "=&r"(d[2]), "=&r"(d[3]), "=&r"(bw)
        : "r"(s[0]), "r"(s[1]), "r"(s[2]), "r"(s[3]), "r"(c), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]));
#pragma unroll
    for (int j = 0; j < 4; ++j) r[j] = bw ? s[j] : d[j];
}

template <> __device__ __forceinline__ void ptx_sub_mod<4>(uint32_t (&r)[4], const uint32_t (&a)[4], const uint32_t (&b)[4], const uint32_t (&p)[4]) {
    uint32_t d[4], mask, q[4];
    asm(
        "sub.cc.u32 %0, %5, %9;\n\t"
        "subc.cc.u32 %1, %6, %10;\n\t"
        "subc.cc.u32 %2, %7, %11;\n\t"
        "subc.cc.u32 %3, %8, %12;\n\t"
        "subc.u32 %4, 0, 0;"
        : "=&r"(d[0]), "=&r"(d[1]), "=&r"(d[2]), "=&r"(d[3]), "=&r"(mask)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]));
#pragma unroll
    for (int j = 0; j < 4; ++j) q[j] = p[j] & mask;
    asm(
        "add.cc.u32 %0, %4, %8;\n\t"
        "addc.cc.u32 %1, %5, %9;\n\t"
        "addc.cc.u32 %2, %6, %10;\n\t"
        "addc.u32 %3, %7, %11;"
        : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3])
        : "r"(d[0]), "r"(d[1]), "r"(d[2]), "r"(d[3]), "r"(q[0]), "r"(q[1]), "r"(q[2]), "r"(q[3]));
}

// ---------------- L = 8 ----------------
template <> __device__ __forceinline__ void ptx_mont_mul<8>(uint32_t (&r)[8], const uint32_t (&a)[8], const uint32_t (&b)[8], const uint32_t (&p)[8], uint32_t np) {
    uint32_t t[10];
    asm(
        "mul.lo.u32 %0, %9, %17;\n\t"
        "mul.lo.u32 %1, %10, %17;\n\t"
        "mul.lo.u32 %2, %11, %17;\n\t"
        "mul.lo.u32 %3, %12, %17;\n\t"
        "mul.lo.u32 %4, %13, %17;\n\t"
        "mul.lo.u32 %5, %14, %17;\n\t"
        "mul.lo.u32 %6, %15, %17;\n\t"
        "mul.lo.u32 %7, %16, %17;\n\t"
        "mov.u32 %8, 0;"
        : "=&r"(t[0]), "=&r"(t[1]), "=&r"(t[2]), "=&r"(t[3]), "=&r"(t[4]), "=&r"(t[5]), "=&r"(t[6]), "=&r"(t[7]), "=&r"(t[8])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b[0]));
    asm(
        "mad.hi.cc.u32 %1, %9, %17, %1;\n\t"
        "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"
        "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"
        "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"
        "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"
        "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"
        "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"
        "madc.hi.u32 %8, %16, %17, %8;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b[0]));
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (i > 0) {
      asm(
          "mad.lo.cc.u32 %0, %9, %17, %0;\n\t"
          "madc.lo.cc.u32 %1, %10, %17, %1;\n\t"
          "madc.lo.cc.u32 %2, %11, %17, %2;\n\t"
          "madc.lo.cc.u32 %3, %12, %17, %3;\n\t"
          "madc.lo.cc.u32 %4, %13, %17, %4;\n\t"
          "madc.lo.cc.u32 %5, %14, %17, %5;\n\t"
          "madc.lo.cc.u32 %6, %15, %17, %6;\n\t"
          "madc.lo.cc.u32 %7, %16, %17, %7;\n\t"
          "addc.u32 %8, %8, 0;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8])
          : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b[i]));
      asm(
          "mad.hi.cc.u32 %1, %9, %17, %1;\n\t"
          "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"
          "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"
          "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"
          "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"
          "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"
          "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"
          "madc.hi.u32 %8, %16, %17, %8;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8])
          : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b[i]));
      }
      const uint32_t m = t[0] * np;
      asm(
          "mad.lo.cc.u32 %0, %18, %10, %0;\n\t"
          "madc.lo.cc.u32 %1, %18, %11, %1;\n\t"
          "madc.lo.cc.u32 %2, %18, %12, %2;\n\t"
          "madc.lo.cc.u32 %3, %18, %13, %3;\n\t"
          "madc.lo.cc.u32 %4, %18, %14, %4;\n\t"
          "madc.lo.cc.u32 %5, %18, %15, %5;\n\t"
          "madc.lo.cc.u32 %6, %18, %16, %6;\n\t"
          "madc.lo.cc.u32 %7, %18, %17, %7;\n\t"
          "addc.cc.u32 %8, %8, 0;\n\t"
          "addc.u32 %9, 0, 0;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8]), "=&r"(t[9])
          : "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]), "r"(m));
      asm(
          "mad.hi.cc.u32 %1, %18, %10, %1;\n\t"
          "madc.hi.cc.u32 %2, %18, %11, %2;\n\t"
          "madc.hi.cc.u32 %3, %18, %12, %3;\n\t"
          "madc.hi.cc.u32 %4, %18, %13, %4;\n\t"
          "madc.hi.cc.u32 %5, %18, %14, %5;\n\t"
          "madc.hi.cc.u32 %6, %18, %15, %6;\n\t"
          "madc.hi.cc.u32 %7, %18, %16, %7;\n\t"
          "madc.hi.cc.u32 %8, %18, %17, %8;\n\t"
          "addc.u32 %9, %9, 0;"
          : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]), "+r"(t[8]), "+r"(t[9])
          : "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]), "r"(m));
#pragma unroll
      for (int j = 0; j <= 8; ++j) t[j] = t[j + 1];
    }
    uint32_t d[8], bw;
    asm(
        "sub.cc.u32 %0, %9, %18;\n\t"
        "subc.cc.u32 %1, %10, %19;\n\t"
        "subc.cc.u32 %2, %11, %20;\n\t"
        "subc.cc.u32 %3, %12, %21;\n\t"
        "subc.cc.u32 %4, %13, %22;\n\t"
        "subc.cc.u32 %5, %14, %23;\n\t"
        "subc.cc.u32 %6, %15, %24;\n\t"
        "subc.cc.u32 %7, %16, %25;\n\t"
        "subc.u32 %8, %17, 0;"
        : "=&r"(d[0]), "=&r"(d[1]), "=&r"(d[2]), "=&r"(d[3]), "=&r"(d[4]), "=&r"(d[5]), "=&r"(d[6]), "=&r"(d[7]), "=&r"(bw)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]), "r"(t[8]), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]));
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = bw ? t[j] : d[j];
}

template <> __device__ __forceinline__ void ptx_add_mod<8>(uint32_t (&r)[8], const uint32_t (&a)[8], const uint32_t (&b)[8], const uint32_t (&p)[8]) {
    uint32_t s[8], d[8], c, bw;
    asm(
        "add.cc.u32 %0, %9, %17;\n\t"
        "addc.cc.u32 %1, %10, %18;\n\t"
        "addc.cc.u32 %2, %11, %19;\n\t"
        "addc.cc.u32 %3, %12, %20;\n\t"
        "addc.cc.u32 %4, %13, %21;\n\t"
        "addc.cc.u32 %5, %14, %22;\n\t"
        "addc.cc.u32 %6, %15, %23;\n\t"
        "addc.cc.u32 %7, %16, %24;\n\t"
        "addc.u32 %8, 0, 0;"
        : "=&r"(s[0]), "=&r"(s[1]), "=&r"(s[2]), "=&r"(s[3]), "=&r"(s[4]), "=&r"(s[5]), "=&r"(s[6]), "=&r"(s[7]), "=&r"(c)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
    asm(
        "sub.cc.u32 %0, %9, %18;\n\t"
        "subc.cc.u32 %1, %10, %19;\n\t"
        "subc.cc.u32 %2, %11, %20;\n\t"
        "subc.cc.u32 %3, %12, %21;\n\t"
        "subc.cc.u32 %4, %13, %22;\n\t"
        "subc.cc.u32 %5, %14, %23;\n\t"
        "subc.cc.u32 %6, %15, %24;\n\t"
        "subc.cc.u32 %7, %16, %25;\n\t"
        "subc.u32 %8, %17, 0;"
        : "=&r"(d[0]), "=&r"(d[1]), "=&r"(d[2]), "=&r"(d[3]), "=&r"(d[4]), "=&r"(d[5]), "=&r"(d[6]), "=&r"(d[7]), "=&r"(bw)
        : "r"(s[0]), "r"(s[1]), "r"(s[2]), "r"(s[3]), "r"(s[4]), "r"(s[5]), "r"(s[6]), "r"(s[7]), "r"(c), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]));
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = bw ? s[j] : d[j];
}

template <> __device__ __forceinline__ void ptx_sub_mod<8>(uint32_t (&r)[8], const uint32_t (&a)[8], const uint32_t (&b)[8], const uint32_t (&p)[8]) {
    uint32_t d[8], mask, q[8];
    asm(
        "sub.cc.u32 %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32 %8, 0, 0;"
        : "=&r"(d[0]), "=&r"(d[1]), "=&r"(d[2]), "=&r"(d[3]), "=&r"(d[4]), "=&r"(d[5]), "=&r"(d[6]), "=&r"(d[7]), "=&r"(mask)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
#pragma unroll
    for (int j = 0; j < 8; ++j) q[j] = p[j] & mask;
    asm(
        "add.cc.u32 %0, %8, %16;\n\t"
        "addc.cc.u32 %1, %9, %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.u32 %7, %15, %23;"
        : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]), "=&r"(r[6]), "=&r"(r[7])
        : "r"(d[0]), "r"(d[1]), "r"(d[2]), "r"(d[3]), "r"(d[4]), "r"(d[5]), "r"(d[6]), "r"(d[7]), "r"(q[0]), "r"(q[1]), "r"(q[2]), "r"(q[3]), "r"(q[4]), "r"(q[5]), "r"(q[6]), "r"(q[7]));
}

