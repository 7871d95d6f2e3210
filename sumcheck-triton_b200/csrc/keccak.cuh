// SHA3-256 on the device, computed by one warp.
//
// Written from FIPS 202 (SHA-3 Standard, NIST 2015): Keccak-f[1600] is 24 rounds of
// theta, rho, pi, chi, iota on a 5x5 array of 64-bit lanes; SHA3-256 absorbs 136-byte
// blocks (rate 1088 bits) after padding the message with 0x06 ... 0x80.
//
// Layout: lane i < 25 of the warp holds state word A[x + 5y] (x = i % 5, y = i / 5).
// Column parities, the pi permutation and chi's neighbours are warp shuffles, so the state
// never leaves registers and costs each thread two registers. The rho offsets and round
// constants are computed at compile time from the standard's own definitions (section
// 3.2.2: offsets (t + 1)(t + 2)/2 along the (x, y) -> (y, 2x + 3y) walk; section 3.2.5: the
// rc LFSR), not typed in.
#pragma once
#include <cstdint>

namespace sc {

struct KeccakConsts {
  uint32_t rot[25];
  uint64_t rc[24];
};

constexpr bool keccak_rc_bit(int t) {
  // FIPS 202 Algorithm 5. Bit k of r is R[k]; R starts as 10000000 (R[0] = 1).
  if (t % 255 == 0) return true;
  unsigned r = 1;
  for (int i = 1; i <= t % 255; ++i) {
    r <<= 1;                     // R = 0 || R, so R[8] is the old R[7]
    if (r & 0x100) r ^= 0x171;   // R[0], R[4], R[5], R[6] ^= R[8]; clears R[8]
    r &= 0xFF;                   // Trunc_8
  }
  return (r & 1) != 0;
}

constexpr KeccakConsts make_keccak_consts() {
  KeccakConsts k{};
  k.rot[0] = 0;
  int x = 1, y = 0;
  for (int t = 0; t < 24; ++t) {
    k.rot[x + 5 * y] = static_cast<uint32_t>(((t + 1) * (t + 2) / 2) % 64);
    int nx = y, ny = (2 * x + 3 * y) % 5;
    x = nx;
    y = ny;
  }
  for (int ir = 0; ir < 24; ++ir) {
    uint64_t rc = 0;
    for (int j = 0; j <= 6; ++j) {
      if (keccak_rc_bit(j + 7 * ir)) rc |= uint64_t{1} << ((1 << j) - 1);
    }
    k.rc[ir] = rc;
  }
  return k;
}

static __constant__ KeccakConsts kKeccak = make_keccak_consts();

__device__ __forceinline__ uint64_t rotl64(uint64_t v, uint32_t r) {
  return (v << r) | (v >> ((64u - r) & 63u));
}

// Keccak-f[1600] on the warp-distributed state (all 32 lanes must call).
__device__ __forceinline__ void keccak_f1600_warp(uint64_t& a, int lane) {
  const int x = lane % 5, y = (lane / 5) % 5;
  const int row = 5 * y;
  const uint32_t rot = lane < 25 ? kKeccak.rot[lane] : 0u;
  // pi (FIPS 202 3.2.3): A'[x, y] = A[(x + 3y) mod 5, x]
  const int src_pi = (x + 3 * y) % 5 + 5 * x;
#pragma unroll 1
  for (int ir = 0; ir < 24; ++ir) {
    // theta
    uint64_t c = a;
#pragma unroll
    for (int k = 1; k < 5; ++k) c ^= __shfl_sync(0xffffffffu, a, x + 5 * ((y + k) % 5));
    const uint64_t cm = __shfl_sync(0xffffffffu, c, (x + 4) % 5 + row);
    const uint64_t cp = __shfl_sync(0xffffffffu, c, (x + 1) % 5 + row);
    a ^= cm ^ rotl64(cp, 1);
    // rho then pi
    const uint64_t b = __shfl_sync(0xffffffffu, rotl64(a, rot), src_pi);
    // chi
    const uint64_t b1 = __shfl_sync(0xffffffffu, b, (x + 1) % 5 + row);
    const uint64_t b2 = __shfl_sync(0xffffffffu, b, (x + 2) % 5 + row);
    a = b ^ (~b1 & b2);
    // iota
    if (lane == 0) a ^= kKeccak.rc[ir];
  }
  if (lane >= 25) a = 0;
}

// SHA3-256 of msg[0..len) held in shared memory. The buffer must have room for the padding
// (len rounded up to a multiple of 136 bytes) and be 8-byte aligned; it is padded in place.
// Every lane of the calling warp gets the 32-byte digest as 8 little-endian words.
__device__ __forceinline__ void sha3_256_warp(uint8_t* msg, int len, uint32_t (&digest)[8]) {
  const int lane = threadIdx.x & 31;
  constexpr int kRate = 136;
  const int nblocks = len / kRate + 1;
  const int padded = nblocks * kRate;
  for (int i = len + lane; i < padded; i += 32) msg[i] = 0;
  __syncwarp();
  if (lane == 0) {
    msg[len] ^= 0x06;
    msg[padded - 1] ^= 0x80;
  }
  __syncwarp();
  uint64_t a = 0;
  const uint64_t* m64 = reinterpret_cast<const uint64_t*>(msg);
  for (int b = 0; b < nblocks; ++b) {
    if (lane < kRate / 8) a ^= m64[b * (kRate / 8) + lane];
    keccak_f1600_warp(a, lane);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint64_t w = __shfl_sync(0xffffffffu, a, i);
    digest[2 * i] = static_cast<uint32_t>(w);
    digest[2 * i + 1] = static_cast<uint32_t>(w >> 32);
  }
}

}  // namespace sc
