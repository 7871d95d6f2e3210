// Table generation and Montgomery conversion kernels.
//
// Generators (one element per thread; the same definitions are restated on the CPU by the
// oracle's uniform_table / bernoulli_table / arith_table):
//   uniform    key_k = mix(seed ^ mix(k + 0x632BE59BD9B4E019)); draw a of element i takes
//              64-bit words mix(key_k + (i << 8 | a << 2 | w)), w = 0..ceil(L/2)-1, as its
//              limbs (low word first); keeps the low bitlen(p) bits; accepts the first
//              draw below p (a < 64; else the last draw minus p, which is below p).
//              mix(x) is SplitMix64's output function applied to x + 0x9E3779B97F4A7C15.
//   bernoulli  low bit of draw 0's first word.
//   arith      the reference's fill, (seed + 7919 (v + 1) + 104729 (i + 1)) mod p
//              (cuda/src/field_sumcheck.cu:123-128, :593-611).
// All are written in Montgomery form (times R^2, then one Montgomery product).
#pragma once
#include <cstdint>

#include "field.cuh"

namespace sc {

struct TableGenArgs {
  int32_t num_tables;
  int32_t pad;
  uint64_t entries;
  uint64_t seed;
  uint64_t p_u64;            // p when p < 2^64, else 0
  uint32_t mask[kMaxLimbs];  // low bitlen(p) bits, per limb
  uint32_t r2[kMaxLimbs];
  int32_t kinds[32];
};

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t table_key(uint64_t seed, int table) {
  return splitmix64(seed ^ splitmix64(static_cast<uint64_t>(table) + 0x632BE59BD9B4E019ull));
}

template <int L>
__device__ __forceinline__ void draw_words(uint64_t key, uint64_t idx, int attempt, uint32_t (&x)[L]) {
#pragma unroll
  for (int w = 0; w < (L + 1) / 2; ++w) {
    const uint64_t z = splitmix64(key + ((idx << 8) | static_cast<uint64_t>((attempt << 2) | w)));
    x[2 * w] = static_cast<uint32_t>(z);
    if (2 * w + 1 < L) x[2 * w + 1] = static_cast<uint32_t>(z >> 32);
  }
}

template <int L>
__device__ __forceinline__ bool below(const uint32_t (&x)[L], const uint32_t (&p)[L]) {
#pragma unroll
  for (int i = L - 1; i >= 0; --i)
    if (x[i] != p[i]) return x[i] < p[i];
  return false;
}

template <int L>
__global__ void generate_tables_kernel(const TableGenArgs G, const FieldParams<L> F, uint32_t* out) {
  const uint64_t total = G.entries * static_cast<uint64_t>(G.num_tables);
  for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < total;
       g += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(g / G.entries);
    const uint64_t i = g - static_cast<uint64_t>(k) * G.entries;
    const int kind = G.kinds[k];
    Fe<L> x = fe_zero<L>();
    if (kind == 0) {
      const uint64_t key = table_key(G.seed, k);
      bool ok = false;
      for (int a = 0; a < 64 && !ok; ++a) {
        draw_words<L>(key, i, a, x.w);
#pragma unroll
        for (int l = 0; l < L; ++l) x.w[l] &= G.mask[l];
        ok = below<L>(x.w, F.p);
      }
      if (!ok) {  // last draw minus p (masked draws are below 2p)
        uint32_t r[L];
        ptx_sub_mod<L>(r, x.w, F.p, F.p);
#pragma unroll
        for (int l = 0; l < L; ++l) x.w[l] = r[l];
      }
    } else if (kind == 1) {
      uint32_t w[L];
      draw_words<L>(table_key(G.seed, k), i, 0, w);
      x.w[0] = w[0] & 1u;
    } else {
      const uint64_t v = static_cast<uint64_t>(kind - 2);
      uint64_t s = (G.seed & 0xFFFFFFFFull) + 7919ull * (v + 1) + 104729ull * (i + 1);
      if (G.p_u64) s %= G.p_u64;
      x.w[0] = static_cast<uint32_t>(s);
      if (L > 1) x.w[1] = static_cast<uint32_t>(s >> 32);
    }
    Fe<L> r2;
#pragma unroll
    for (int l = 0; l < L; ++l) r2.w[l] = G.r2[l];
    const Fe<L> m = fe_mul(x, r2, F);
#pragma unroll
    for (int l = 0; l < L; ++l) out[(static_cast<uint64_t>(k) * L + l) * G.entries + i] = m.w[l];
  }
}

// In place: x -> x * factor / R for every element (factor = R^2: to Montgomery; 1: back).
template <int L>
__global__ void convert_tables_kernel(uint32_t* tables, uint64_t entries, int num_tables, const Fe<L> factor,
                                      const FieldParams<L> F) {
  const uint64_t total = entries * static_cast<uint64_t>(num_tables);
  for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < total;
       g += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t k = g / entries, i = g - k * entries;
    Fe<L> x;
#pragma unroll
    for (int l = 0; l < L; ++l) x.w[l] = tables[(k * L + l) * entries + i];
    const Fe<L> m = fe_mul(x, factor, F);
#pragma unroll
    for (int l = 0; l < L; ++l) tables[(k * L + l) * entries + i] = m.w[l];
  }
}

// out[i] = a[i] op b[i] over element-major arrays (the prover's own arithmetic, for tests).
template <int L>
__global__ void field_apply_kernel(int op, const uint32_t* a, const uint32_t* b, uint32_t* out, uint64_t count,
                                   const FieldParams<L> F) {
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    Fe<L> x, y;
#pragma unroll
    for (int l = 0; l < L; ++l) {
      x.w[l] = a[i * L + l];
      y.w[l] = b[i * L + l];
    }
    const Fe<L> r = op == 0 ? fe_mul(x, y, F) : (op == 1 ? fe_add(x, y, F) : fe_sub(x, y, F));
#pragma unroll
    for (int l = 0; l < L; ++l) out[i * L + l] = r.w[l];
  }
}

// Integer multiply-add throughput probe: every thread runs 8 independent chains of
// mad.lo / mad.hi (the instruction pair of the Montgomery product), so the count of
// multiply-adds is exact: iters x 8 chains x 2 per thread.
static __global__ void imad_probe_kernel(uint32_t* sink, int iters, uint32_t seed) {
  uint32_t a[8], b[8];
  const uint32_t x = seed ^ threadIdx.x, y = seed * 0x9E3779B9u + blockIdx.x;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    a[c] = x + c;
    b[c] = y ^ c;
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      asm volatile("mad.lo.u32 %0, %2, %3, %0;\n\tmad.hi.u32 %1, %2, %3, %1;"
                   : "+r"(a[c]), "+r"(b[c])
                   : "r"(x), "r"(y + c));
    }
  }
  uint32_t acc = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) acc ^= a[c] ^ b[c];
  if (acc == 0x12345678u) sink[0] = acc;  // keeps the chains live
}

}  // namespace sc
