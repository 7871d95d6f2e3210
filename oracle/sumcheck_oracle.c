/*
 * CPU oracle of the SumCheck prover path in C -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg load this library
 * (oracle/_build/liboracle.so), and only as the checker or the timed CPU baseline.
 *
 * It restates the same algorithm as oracle/oracle.py, for sizes Python big integers cannot
 * reach, and is pinned against it (tests/test_c_oracle.py):
 *   - the round loop of the reference's sumcheck_reference (src/zkduel/reference.py:44-110):
 *     g(0), g(1) from evens and odds, g(t >= 2) by adding the difference, then the fold
 *     e + r (o - e);
 *   - the transcript rule of cuda/src/field_sumcheck.cu:857-907 (SHA3-256 over
 *     "zkduel:field-sweep:v1" || u32le(round) || u32le(Montgomery limbs of g(0..d)), digest
 *     read little-endian, reduced mod p), here with a plain Keccak-f[1600] from FIPS 202;
 *   - the checksum sum (i + 1) limb_i of field_sumcheck.cu:1046-1049;
 *   - the project's table generators (csrc/tables.cuh), and the reference's arithmetic
 *     progression fill (field_sumcheck.cu:123-128).
 * Arithmetic: Montgomery form with a textbook fully carried CIOS (L + 2 words), so it does
 * not share the device routine's (L + 1)-word shortcut. Rounds run on `threads` POSIX
 * threads (split over pairs), which is also how the CPU baseline uses every host core.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAXL 8
#define MAXP 8
#define MAXK 32

typedef struct {
  int L;
  uint32_t p[MAXL];
  uint32_t np;
  uint32_t r2[MAXL];
  uint32_t one[MAXL];
} field_t;

/* ---------------------------------------------------------------- arithmetic */

static int geq(const field_t* f, const uint32_t* a, const uint32_t* b) {
  for (int i = f->L - 1; i >= 0; --i)
    if (a[i] != b[i]) return a[i] > b[i];
  return 1;
}

static uint32_t sub_raw(int L, const uint32_t* a, const uint32_t* b, uint32_t* r) {
  uint64_t br = 0;
  for (int i = 0; i < L; ++i) {
    uint64_t d = (uint64_t)a[i] - b[i] - br;
    r[i] = (uint32_t)d;
    br = (d >> 63) & 1;
  }
  return (uint32_t)br;
}

static uint32_t add_raw(int L, const uint32_t* a, const uint32_t* b, uint32_t* r) {
  uint64_t c = 0;
  for (int i = 0; i < L; ++i) {
    uint64_t s = (uint64_t)a[i] + b[i] + c;
    r[i] = (uint32_t)s;
    c = s >> 32;
  }
  return (uint32_t)c;
}

static void f_add(const field_t* f, const uint32_t* a, const uint32_t* b, uint32_t* r) {
  uint32_t s[MAXL];
  uint32_t c = add_raw(f->L, a, b, s);
  if (c || geq(f, s, f->p)) sub_raw(f->L, s, f->p, s);
  memcpy(r, s, 4 * f->L);
}

static void f_sub(const field_t* f, const uint32_t* a, const uint32_t* b, uint32_t* r) {
  uint32_t d[MAXL];
  if (sub_raw(f->L, a, b, d)) add_raw(f->L, d, f->p, d);
  memcpy(r, d, 4 * f->L);
}

static void f_mul(const field_t* f, const uint32_t* a, const uint32_t* b, uint32_t* r) {
  const int L = f->L;
  uint32_t t[MAXL + 2];
  memset(t, 0, sizeof(t));
  for (int i = 0; i < L; ++i) {
    uint64_t c = 0;
    for (int j = 0; j < L; ++j) {
      uint64_t uv = (uint64_t)t[j] + (uint64_t)a[j] * b[i] + c;
      t[j] = (uint32_t)uv;
      c = uv >> 32;
    }
    uint64_t s = (uint64_t)t[L] + c;
    t[L] = (uint32_t)s;
    t[L + 1] = (uint32_t)(s >> 32);
    uint32_t m = t[0] * f->np;
    c = 0;
    for (int j = 0; j < L; ++j) {
      uint64_t uv = (uint64_t)t[j] + (uint64_t)m * f->p[j] + c;
      t[j] = (uint32_t)uv;
      c = uv >> 32;
    }
    s = (uint64_t)t[L] + c;
    t[L] = (uint32_t)s;
    t[L + 1] += (uint32_t)(s >> 32);
    for (int j = 0; j <= L; ++j) t[j] = t[j + 1];
    t[L + 1] = 0;
  }
  if (t[L] || geq(f, t, f->p)) sub_raw(L, t, f->p, t);
  memcpy(r, t, 4 * L);
}

static void f_dbl(const field_t* f, uint32_t* a) { f_add(f, a, a, a); }

static int field_setup(field_t* f, int L, const uint32_t* p) {
  memset(f, 0, sizeof(*f));
  f->L = L;
  memcpy(f->p, p, 4 * L);
  uint32_t inv = 1;
  for (int i = 0; i < 5; ++i) inv *= 2u - p[0] * inv;
  f->np = 0u - inv;
  uint32_t x[MAXL] = {0};
  x[0] = 1;
  for (int i = 0; i < 32 * L; ++i) f_dbl(f, x);
  memcpy(f->one, x, 4 * L);
  for (int i = 0; i < 32 * L; ++i) f_dbl(f, x);
  memcpy(f->r2, x, 4 * L);
  return 0;
}

/* canonical small value v (< 2^64) -> Montgomery */
static void mont_u64(const field_t* f, uint64_t v, uint32_t* out) {
  uint32_t acc[MAXL] = {0};
  for (int b = 63; b >= 0; --b) {
    f_dbl(f, acc);
    if ((v >> b) & 1) {
      uint32_t one[MAXL] = {0};
      one[0] = 1;
      f_add(f, acc, one, acc);
    }
  }
  f_mul(f, acc, f->r2, out);
}

static void mont_pow(const field_t* f, const uint32_t* base, const uint32_t* e, uint32_t* out) {
  uint32_t acc[MAXL];
  memcpy(acc, f->one, 4 * f->L);
  for (int w = f->L - 1; w >= 0; --w)
    for (int b = 31; b >= 0; --b) {
      f_mul(f, acc, acc, acc);
      if ((e[w] >> b) & 1u) f_mul(f, acc, base, acc);
    }
  memcpy(out, acc, 4 * f->L);
}

/* ---------------------------------------------------------------- SHA3-256 (FIPS 202) */

static const uint64_t RC[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808AULL, 0x8000000080008000ULL,
    0x000000000000808BULL, 0x0000000080000001ULL, 0x8000000080008081ULL, 0x8000000000008009ULL,
    0x000000000000008AULL, 0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000AULL,
    0x000000008000808BULL, 0x800000000000008BULL, 0x8000000000008089ULL, 0x8000000000008003ULL,
    0x8000000000008002ULL, 0x8000000000000080ULL, 0x000000000000800AULL, 0x800000008000000AULL,
    0x8000000080008081ULL, 0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};

static uint64_t rotl(uint64_t x, int r) { return r ? (x << r) | (x >> (64 - r)) : x; }

static void keccak_f(uint64_t A[25]) {
  int rot[25];
  /* rho offsets from FIPS 202 3.2.2 */
  rot[0] = 0;
  int x = 1, y = 0;
  for (int t = 0; t < 24; ++t) {
    rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
    int nx = y, ny = (2 * x + 3 * y) % 5;
    x = nx;
    y = ny;
  }
  for (int ir = 0; ir < 24; ++ir) {
    uint64_t C[5], D[5], B[25];
    for (int i = 0; i < 5; ++i) C[i] = A[i] ^ A[i + 5] ^ A[i + 10] ^ A[i + 15] ^ A[i + 20];
    for (int i = 0; i < 5; ++i) D[i] = C[(i + 4) % 5] ^ rotl(C[(i + 1) % 5], 1);
    for (int i = 0; i < 25; ++i) A[i] ^= D[i % 5];
    for (int xx = 0; xx < 5; ++xx)
      for (int yy = 0; yy < 5; ++yy) B[yy + 5 * ((2 * xx + 3 * yy) % 5)] = rotl(A[xx + 5 * yy], rot[xx + 5 * yy]);
    for (int yy = 0; yy < 5; ++yy)
      for (int xx = 0; xx < 5; ++xx)
        A[xx + 5 * yy] = B[xx + 5 * yy] ^ (~B[(xx + 1) % 5 + 5 * yy] & B[(xx + 2) % 5 + 5 * yy]);
    A[0] ^= RC[ir];
  }
}

void oracle_sha3_256(const uint8_t* msg, size_t len, uint8_t out[32]) {
  uint64_t A[25];
  memset(A, 0, sizeof(A));
  const size_t rate = 136;
  uint8_t block[136];
  size_t off = 0;
  for (;;) {
    size_t take = len - off < rate ? len - off : rate;
    memset(block, 0, rate);
    memcpy(block, msg + off, take);
    int last = take < rate;
    if (last) {
      block[take] ^= 0x06;
      block[rate - 1] ^= 0x80;
    }
    for (int i = 0; i < 17; ++i) {
      uint64_t w = 0;
      for (int b = 0; b < 8; ++b) w |= (uint64_t)block[8 * i + b] << (8 * b);
      A[i] ^= w;
    }
    keccak_f(A);
    off += take;
    if (last) break;
  }
  for (int i = 0; i < 32; ++i) out[i] = (uint8_t)(A[i / 8] >> (8 * (i % 8)));
}

/* ---------------------------------------------------------------- generators */

static uint64_t mix(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* What the generators need of a modulus: its bit mask per limb and, when p < 2^64, p. */
typedef struct {
  int L;
  uint32_t p[MAXL];
  uint32_t mask[MAXL];
  uint64_t p64;
  uint64_t seed;
} gen_t;

static void gen_setup(gen_t* g, int L, const uint32_t* p, uint64_t seed) {
  memset(g, 0, sizeof(*g));
  g->L = L;
  memcpy(g->p, p, 4 * L);
  g->seed = seed;
  int bits = 0;
  for (int l = L - 1; l >= 0 && !bits; --l)
    if (p[l]) bits = 32 * l + (32 - __builtin_clz(p[l]));
  for (int l = 0; l < L; ++l) {
    int lo = 32 * l;
    g->mask[l] = bits >= lo + 32 ? 0xFFFFFFFFu : (bits <= lo ? 0u : ((1u << (bits - lo)) - 1u));
  }
  int fits64 = 1;
  for (int l = 2; l < L; ++l) fits64 = fits64 && p[l] == 0;
  g->p64 = fits64 ? (((uint64_t)(L > 1 ? p[1] : 0)) << 32) | p[0] : 0;
}

static uint64_t gen_key(const gen_t* g, int k) { return mix(g->seed ^ mix((uint64_t)k + 0x632BE59BD9B4E019ULL)); }

/* Entry i of table k (canonical limbs): kind 0 uniform, 1 bernoulli, 2 + v arith. */
static void gen_entry(const gen_t* g, const field_t* f, int kind, uint64_t key, uint64_t i, uint32_t* x) {
  const int L = g->L;
  memset(x, 0, 4 * MAXL);
  if (kind == 0) {
    int ok = 0;
    for (int a = 0; a < 64 && !ok; ++a) {
      for (int w = 0; w < (L + 1) / 2; ++w) {
        uint64_t z = mix(key + ((i << 8) | (uint64_t)((a << 2) | w)));
        x[2 * w] = (uint32_t)z;
        if (2 * w + 1 < L) x[2 * w + 1] = (uint32_t)(z >> 32);
      }
      for (int l = 0; l < L; ++l) x[l] &= g->mask[l];
      ok = !geq(f, x, g->p);
    }
    if (!ok) sub_raw(L, x, g->p, x);
  } else if (kind == 1) {
    x[0] = (uint32_t)mix(key + (i << 8)) & 1u;
  } else {
    uint64_t v = (uint64_t)(kind - 2);
    uint64_t s = (g->seed & 0xFFFFFFFFULL) + 7919ULL * (v + 1) + 104729ULL * (i + 1);
    if (g->p64) s %= g->p64;
    x[0] = (uint32_t)s;
    if (L > 1) x[1] = (uint32_t)(s >> 32);
  }
}

/* Canonical tables, limb-planar (K, L, 2^n): kinds 0 uniform, 1 bernoulli, 2 + v arith. */
int oracle_generate(int L, const uint32_t* p, int K, int n, const int32_t* kinds, uint64_t seed, uint32_t* out) {
  const uint64_t N = (uint64_t)1 << n;
  field_t f;
  field_setup(&f, L, p);
  gen_t g;
  gen_setup(&g, L, p, seed);
  for (int k = 0; k < K; ++k) {
    const uint64_t key = gen_key(&g, k);
    for (uint64_t i = 0; i < N; ++i) {
      uint32_t x[MAXL];
      gen_entry(&g, &f, kinds[k], key, i, x);
      for (int l = 0; l < L; ++l) out[((uint64_t)k * L + l) * N + i] = x[l];
    }
  }
  return 0;
}

/* ---------------------------------------------------------------- prover */

typedef struct {
  const field_t* f;
  int K, T, d;
  const int32_t* lens;
  const int32_t* offs;
  const int32_t* flat;
  const uint32_t* cm; /* T x L Montgomery coefficients */
  const uint32_t* cur; /* K x N x L element-major, Montgomery (NULL: generate, see gen) */
  uint32_t* nxt;
  const gen_t* gen;    /* round 0 of a seeded proof: entries generated on the fly */
  const int32_t* kinds;
  uint64_t keys[MAXK];
  uint64_t N;          /* entries per table in cur */
  uint64_t lo, hi;     /* pair range */
  uint32_t r[MAXL];
  uint32_t acc[MAXP][MAXL];
  int phase; /* 0 eval, 1 fold */
} job_t;

/* Entries 2i and 2i + 1 of table k, Montgomery, into e[0..2L). */
static const uint32_t* pair_at(const job_t* J, int k, uint64_t i, uint32_t* buf) {
  const int L = J->f->L;
  if (J->cur) return J->cur + ((uint64_t)k * J->N + 2 * i) * L;
  for (int h = 0; h < 2; ++h) {
    uint32_t x[MAXL];
    gen_entry(J->gen, J->f, J->kinds[k], J->keys[k], 2 * i + h, x);
    f_mul(J->f, x, J->f->r2, buf + h * L);
  }
  return buf;
}

static void* run_job(void* arg) {
  job_t* J = (job_t*)arg;
  const field_t* f = J->f;
  const int L = f->L, K = J->K;
  uint32_t buf[2 * MAXL];
  if (J->phase == 0) {
    uint32_t v[MAXK][MAXL], df[MAXK][MAXL];
    memset(J->acc, 0, sizeof(J->acc));
    for (uint64_t i = J->lo; i < J->hi; ++i) {
      for (int k = 0; k < K; ++k) {
        const uint32_t* e = pair_at(J, k, i, buf);
        memcpy(v[k], e, 4 * L);
        f_sub(f, e + L, e, df[k]);
      }
      for (int t = 0; t <= J->d; ++t) {
        if (t)
          for (int k = 0; k < K; ++k) f_add(f, v[k], df[k], v[k]);
        uint32_t tot[MAXL] = {0};
        for (int m = 0; m < J->T; ++m) {
          uint32_t prod[MAXL];
          memcpy(prod, J->cm + m * L, 4 * L);
          for (int q = 0; q < J->lens[m]; ++q) f_mul(f, prod, v[J->flat[J->offs[m] + q]], prod);
          f_add(f, tot, prod, tot);
        }
        f_add(f, J->acc[t], tot, J->acc[t]);
      }
    }
  } else {
    const uint64_t half = J->N / 2;
    for (int k = 0; k < K; ++k)
      for (uint64_t i = J->lo; i < J->hi; ++i) {
        const uint32_t* e = pair_at(J, k, i, buf);
        uint32_t d[MAXL], x[MAXL];
        f_sub(f, e + L, e, d);
        f_mul(f, J->r, d, x);
        f_add(f, e, x, J->nxt + ((uint64_t)k * half + i) * L);
      }
  }
  return NULL;
}

static void run_parallel(job_t* jobs, int threads, uint64_t count) {
  pthread_t th[256];
  int created[256] = {0};
  uint64_t per = (count + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    jobs[t].lo = per * t < count ? per * t : count;
    jobs[t].hi = per * (t + 1) < count ? per * (t + 1) : count;
  }
  for (int t = 1; t < threads; ++t)
    if (jobs[t].lo < jobs[t].hi) created[t] = pthread_create(&th[t], NULL, run_job, &jobs[t]) == 0;
  run_job(&jobs[0]);
  for (int t = 1; t < threads; ++t) {
    if (created[t]) pthread_join(th[t], NULL);
    else if (jobs[t].lo < jobs[t].hi) run_job(&jobs[t]);
  }
}

/*
 * tables: canonical, limb-planar (K, L, 2^n); or NULL, and then round 0 generates every
 * entry on the fly from (kinds, seed) -- the same values oracle_generate writes -- so a
 * seeded proof holds only the folded tables (half the entries, Montgomery). mode 0 sha3,
 * 1 fixed (r = 1), 2 explicit (explicit_canon: n x L canonical limbs). Outputs in
 * Montgomery limbs: out_polys n x (d + 1) x L, out_chals n x L, out_finals (1 + K) x L,
 * out_claim0 L.
 */
static int prove_core(int L, const uint32_t* p, int K, int T, const int64_t* coeffs, const int32_t* lens,
                      const int32_t* offs, const int32_t* flat, int n, const uint32_t* tables,
                      const int32_t* kinds, uint64_t seed, int mode, const uint32_t* explicit_canon, int threads,
                      uint32_t* out_polys, uint32_t* out_chals, uint32_t* out_finals, uint32_t* out_claim0,
                      uint64_t* out_checksum) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  if (K > MAXK || L > MAXL || n < 1 || n > 40) return 1;
  field_t f;
  field_setup(&f, L, p);
  gen_t g;
  gen_setup(&g, L, p, seed);
  int d = 0;
  for (int m = 0; m < T; ++m) d = lens[m] > d ? lens[m] : d;
  if (d > MAXP - 1) return 1;
  uint64_t N = (uint64_t)1 << n;
  const uint64_t sizeA = tables ? N : N / 2, sizeB = tables ? N / 2 : (N / 4 > 0 ? N / 4 : 1);
  uint32_t* bufA = (uint32_t*)malloc(sizeof(uint32_t) * K * sizeA * L);
  uint32_t* bufB = (uint32_t*)malloc(sizeof(uint32_t) * K * sizeB * L);
  uint32_t* cm = (uint32_t*)malloc(sizeof(uint32_t) * T * L);
  job_t* jobs = (job_t*)calloc(threads, sizeof(job_t));
  if (!bufA || !bufB || !cm || !jobs) {
    free(bufA);
    free(bufB);
    free(cm);
    free(jobs);
    return 2;
  }
  uint32_t* cur = tables ? bufA : NULL;
  uint32_t* nxt = tables ? bufB : bufA;
  if (tables)
    for (int k = 0; k < K; ++k)
      for (uint64_t i = 0; i < N; ++i) {
        uint32_t x[MAXL];
        for (int l = 0; l < L; ++l) x[l] = tables[((uint64_t)k * L + l) * N + i];
        f_mul(&f, x, f.r2, cur + ((uint64_t)k * N + i) * L);
      }
  for (int m = 0; m < T; ++m) {
    int64_t c = coeffs[m];
    uint64_t mag = c < 0 ? (uint64_t)(-(c + 1)) + 1 : (uint64_t)c;
    mont_u64(&f, mag, cm + m * L);
    if (c < 0) {
      uint32_t z[MAXL] = {0};
      f_sub(&f, z, cm + m * L, cm + m * L);
    }
  }
  uint64_t checksum = 0;
  uint32_t r[MAXL];
  for (int j = 0; j < n; ++j) {
    const uint64_t half = N / 2;
    for (int t = 0; t < threads; ++t) {
      job_t* J = &jobs[t];
      J->f = &f;
      J->K = K;
      J->T = T;
      J->d = d;
      J->lens = lens;
      J->offs = offs;
      J->flat = flat;
      J->cm = cm;
      J->cur = cur;
      J->nxt = nxt;
      J->N = N;
      J->phase = 0;
      J->gen = &g;
      J->kinds = kinds;
      for (int k = 0; k < K && !cur; ++k) J->keys[k] = gen_key(&g, k);
      memset(J->acc, 0, sizeof(J->acc)); /* a job with an empty range contributes zero */
    }
    run_parallel(jobs, half < (uint64_t)threads ? 1 : threads, half);
    uint32_t g[MAXP][MAXL];
    memset(g, 0, sizeof(g));
    int used = half < (uint64_t)threads ? 1 : threads;
    for (int t = 0; t < used; ++t)
      for (int q = 0; q <= d; ++q) f_add(&f, g[q], jobs[t].acc[q], g[q]);
    for (int q = 0; q <= d; ++q)
      for (int l = 0; l < L; ++l) {
        out_polys[((uint64_t)j * (d + 1) + q) * L + l] = g[q][l];
        checksum += (uint64_t)(l + 1) * g[q][l];
      }
    if (j == 0) f_add(&f, g[0], g[1], out_claim0);
    /* challenge */
    if (mode == 0) {
      uint8_t msg[21 + 4 + 4 * MAXP * MAXL];
      memcpy(msg, "zkduel:field-sweep:v1", 21);
      size_t pos = 21;
      uint32_t words[1 + MAXP * MAXL];
      int nw = 0;
      words[nw++] = (uint32_t)j;
      for (int q = 0; q <= d; ++q)
        for (int l = 0; l < L; ++l) words[nw++] = g[q][l];
      for (int w = 0; w < nw; ++w)
        for (int b = 0; b < 4; ++b) msg[pos++] = (uint8_t)(words[w] >> (8 * b));
      uint8_t dig[32];
      oracle_sha3_256(msg, pos, dig);
      /* Horner over 32-bit digest words, most significant first, in canonical form */
      uint32_t acc[MAXL] = {0};
      int small = 1;
      for (int l = 1; l < L; ++l) small = small && p[l] == 0;
      for (int w = 7; w >= 0; --w) {
        for (int b = 0; b < 32; ++b) f_dbl(&f, acc);
        uint32_t word = (uint32_t)dig[4 * w] | ((uint32_t)dig[4 * w + 1] << 8) | ((uint32_t)dig[4 * w + 2] << 16) |
                        ((uint32_t)dig[4 * w + 3] << 24);
        uint32_t x[MAXL] = {0};
        x[0] = small ? word % p[0] : word;
        f_add(&f, acc, x, acc);
      }
      f_mul(&f, acc, f.r2, r);
    } else if (mode == 1) {
      memcpy(r, f.one, 4 * L);
    } else {
      f_mul(&f, explicit_canon + (uint64_t)j * L, f.r2, r);
    }
    memcpy(out_chals + (uint64_t)j * L, r, 4 * L);
    /* fold */
    for (int t = 0; t < threads; ++t) {
      jobs[t].phase = 1;
      memcpy(jobs[t].r, r, 4 * L);
    }
    run_parallel(jobs, half < (uint64_t)threads ? 1 : threads, half);
    if (cur == NULL) { /* round 0 of a seeded proof: T_1 is in bufA, fold into bufB next */
      cur = bufA;
      nxt = bufB;
    } else {
      uint32_t* tmp = cur;
      cur = nxt;
      nxt = tmp;
    }
    N = half;
    if (j == n - 1) {
      /* final claim: Lagrange interpolation of g at r; folded values f_k(r) */
      uint32_t pm2[MAXL];
      uint32_t two[MAXL] = {0};
      two[0] = 2;
      sub_raw(L, p, two, pm2);
      uint32_t total[MAXL] = {0};
      for (int q = 0; q <= d; ++q) {
        uint32_t num[MAXL], den[MAXL], tmpv[MAXL];
        memcpy(num, f.one, 4 * L);
        memcpy(den, f.one, 4 * L);
        for (int s = 0; s <= d; ++s) {
          if (s == q) continue;
          uint32_t sm[MAXL], qm[MAXL];
          mont_u64(&f, (uint64_t)s, sm);
          mont_u64(&f, (uint64_t)q, qm);
          f_sub(&f, r, sm, tmpv);
          f_mul(&f, num, tmpv, num);
          f_sub(&f, qm, sm, tmpv);
          f_mul(&f, den, tmpv, den);
        }
        uint32_t inv[MAXL];
        mont_pow(&f, den, pm2, inv);
        f_mul(&f, num, inv, tmpv);
        f_mul(&f, tmpv, g[q], tmpv);
        f_add(&f, total, tmpv, total);
      }
      memcpy(out_finals, total, 4 * L);
      for (int k = 0; k < K; ++k) memcpy(out_finals + (uint64_t)(1 + k) * L, cur + (uint64_t)k * L, 4 * L);
    }
  }
  *out_checksum = checksum;
  free(bufA);
  free(bufB);
  free(cm);
  free(jobs);
  return 0;
}

int oracle_prove(int L, const uint32_t* p, int K, int T, const int64_t* coeffs, const int32_t* lens,
                 const int32_t* offs, const int32_t* flat, int n, const uint32_t* tables, int mode,
                 const uint32_t* explicit_canon, int threads, uint32_t* out_polys, uint32_t* out_chals,
                 uint32_t* out_finals, uint32_t* out_claim0, uint64_t* out_checksum) {
  if (!tables) return 1;
  return prove_core(L, p, K, T, coeffs, lens, offs, flat, n, tables, NULL, 0, mode, explicit_canon, threads,
                    out_polys, out_chals, out_finals, out_claim0, out_checksum);
}

/* The proof of the seeded tables oracle_generate(L, p, K, n, kinds, seed) would write,
 * without writing them: round 0 generates its entries on the fly (see prove_core). */
int oracle_prove_seeded(int L, const uint32_t* p, int K, int T, const int64_t* coeffs, const int32_t* lens,
                        const int32_t* offs, const int32_t* flat, int n, const int32_t* kinds, uint64_t seed,
                        int mode, const uint32_t* explicit_canon, int threads, uint32_t* out_polys,
                        uint32_t* out_chals, uint32_t* out_finals, uint32_t* out_claim0, uint64_t* out_checksum) {
  if (!kinds) return 1;
  return prove_core(L, p, K, T, coeffs, lens, offs, flat, n, NULL, kinds, seed, mode, explicit_canon, threads,
                    out_polys, out_chals, out_finals, out_claim0, out_checksum);
}
