// Host-side big-integer arithmetic for field set-up (moduli up to 8 limbs).
//
// Used once per field / expression to derive the constants the device needs: R mod p,
// R^2 mod p, Montgomery images of small integers, the digest-reduction table and the
// Lagrange weights. Plain fully-carried CIOS with 64-bit intermediates; nothing here is on
// the proving path.
#pragma once
#include <cstdint>
#include <cstring>
#include <string>

namespace sc {

struct HostField {
  int L = 0;
  uint32_t p[8] = {0};
  uint32_t np = 0;

  // a >= b over L limbs?
  bool geq(const uint32_t* a, const uint32_t* b) const {
    for (int i = L - 1; i >= 0; --i)
      if (a[i] != b[i]) return a[i] > b[i];
    return true;
  }
  // r = a - b (L limbs), returns the borrow
  uint32_t sub_raw(const uint32_t* a, const uint32_t* b, uint32_t* r) const {
    uint64_t br = 0;
    for (int i = 0; i < L; ++i) {
      uint64_t d = static_cast<uint64_t>(a[i]) - b[i] - br;
      r[i] = static_cast<uint32_t>(d);
      br = (d >> 63) & 1;
    }
    return static_cast<uint32_t>(br);
  }
  uint32_t add_raw(const uint32_t* a, const uint32_t* b, uint32_t* r) const {
    uint64_t c = 0;
    for (int i = 0; i < L; ++i) {
      uint64_t s = static_cast<uint64_t>(a[i]) + b[i] + c;
      r[i] = static_cast<uint32_t>(s);
      c = s >> 32;
    }
    return static_cast<uint32_t>(c);
  }
  // a, b < p
  void add(const uint32_t* a, const uint32_t* b, uint32_t* r) const {
    uint32_t s[8];
    uint32_t c = add_raw(a, b, s);
    if (c || geq(s, p)) sub_raw(s, p, s);
    std::memcpy(r, s, 4 * L);
  }
  void sub(const uint32_t* a, const uint32_t* b, uint32_t* r) const {
    uint32_t d[8];
    if (sub_raw(a, b, d)) add_raw(d, p, d);
    std::memcpy(r, d, 4 * L);
  }
  void neg(const uint32_t* a, uint32_t* r) const {
    uint32_t z[8] = {0};
    sub(z, a, r);
  }
  // Montgomery product a b R^-1 mod p, a, b < p, textbook CIOS with L + 2 words.
  void mul(const uint32_t* a, const uint32_t* b, uint32_t* r) const {
    uint32_t t[10] = {0};
    for (int i = 0; i < L; ++i) {
      uint64_t c = 0;
      for (int j = 0; j < L; ++j) {
        uint64_t uv = static_cast<uint64_t>(t[j]) + static_cast<uint64_t>(a[j]) * b[i] + c;
        t[j] = static_cast<uint32_t>(uv);
        c = uv >> 32;
      }
      uint64_t s = static_cast<uint64_t>(t[L]) + c;
      t[L] = static_cast<uint32_t>(s);
      t[L + 1] = static_cast<uint32_t>(s >> 32);
      const uint32_t m = t[0] * np;
      c = 0;
      for (int j = 0; j < L; ++j) {
        uint64_t uv = static_cast<uint64_t>(t[j]) + static_cast<uint64_t>(m) * p[j] + c;
        t[j] = static_cast<uint32_t>(uv);
        c = uv >> 32;
      }
      s = static_cast<uint64_t>(t[L]) + c;
      t[L] = static_cast<uint32_t>(s);
      t[L + 1] += static_cast<uint32_t>(s >> 32);
      for (int j = 0; j <= L; ++j) t[j] = t[j + 1];
      t[L + 1] = 0;
    }
    if (t[L] || geq(t, p)) sub_raw(t, p, t);
    std::memcpy(r, t, 4 * L);
  }
  // 2a mod p
  void dbl(const uint32_t* a, uint32_t* r) const { add(a, a, r); }

  // v mod p for an arbitrary non-negative integer of nwords u32 words (bit-serial).
  void reduce(const uint32_t* v, int nwords, uint32_t* r) const {
    uint32_t acc[8] = {0};
    uint32_t one[8] = {0};
    one[0] = 1;
    uint32_t one_red[8];
    std::memcpy(one_red, one, sizeof(one));
    if (L == 1 && one_red[0] >= p[0]) one_red[0] %= p[0];
    for (int w = nwords - 1; w >= 0; --w) {
      for (int b = 31; b >= 0; --b) {
        dbl(acc, acc);
        if ((v[w] >> b) & 1u) add(acc, one_red, acc);
      }
    }
    std::memcpy(r, acc, 4 * L);
  }
};

}  // namespace sc
