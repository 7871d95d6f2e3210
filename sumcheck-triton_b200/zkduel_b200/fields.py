"""Prime fields of the prover and the guard on their moduli.

The four configured fields are the reference's (``src/zkduel/fields.py:258-294``):
2^32-5, Goldilocks, 2^127-1 and the BLS12-381 scalar field, each held as little-endian
32-bit limbs in Montgomery form (R = 2^(32 L)).

The device multiplication (``csrc/field.cuh``) is a CIOS Montgomery product whose
accumulator between outer iterations is L+1 words. That is exact only when
``(2p - 1) + (p - 1)(2^32 - 1) < 2^(32 (L + 1))`` -- the same contract the reference's
kernels carry (``cuda/src/field_sumcheck.cu:277-319``, guard ``fields.py:118-121``).
``check_montgomery_modulus`` rejects every modulus outside it, with the reference's error
type (``UnsafeModulusError``, a ``ValueError``) and error wording, so a caller that relied
on the reference rejecting a modulus sees the same rejection here.

The reference also runs a randomized stress test after the bound check
(``fields.py:154-187``); the bound is sufficient, so with it holding that test cannot
fire and the set of rejected moduli is the bound alone. ``stress_value`` below is this
project's own generator of carry-heavy operands, used by the device-arithmetic tests.
"""

from __future__ import annotations

import random
from dataclasses import dataclass
from functools import lru_cache

MASK32 = 0xFFFFFFFF
SUPPORTED_LIMBS = (1, 2, 4, 8)
MAX_POINTS = 8  # interpolation points t = 0..7, so degree <= 7 (field_sumcheck.cu:29)


class UnsafeModulusError(ValueError):
    """The device Montgomery multiplication is not exact for this modulus."""


def montgomery_nprime(modulus: int) -> int:
    """-p^-1 mod 2^32, the per-limb Montgomery constant."""
    return (-pow(int(modulus), -1, 1 << 32)) & MASK32


def cios_bound_holds(modulus: int, limbs: int) -> bool:
    """Sufficient condition for the (L+1)-word CIOS product to be exact for a, b < p."""
    p = int(modulus)
    return (2 * p - 1) + (p - 1) * MASK32 < (1 << (32 * (int(limbs) + 1)))


@lru_cache(maxsize=None)
def check_montgomery_modulus(modulus: int, limbs: int, nprime: int) -> None:
    """Raise ``UnsafeModulusError`` unless the device Montgomery product is exact.

    Same rejections, in the same order, as the reference's guard
    (``src/zkduel/fields.py:190-227``): limb count, odd modulus > 2, fits in L limbs,
    nprime, then the CIOS bound.
    """
    p, L, nprime = int(modulus), int(limbs), int(nprime)
    where = f"modulus {p:#x} with {L} x 32-bit limbs"
    if L < 1:
        raise UnsafeModulusError(f"{where}: need at least one limb")
    if p < 3 or p % 2 == 0:
        raise UnsafeModulusError(f"{where}: Montgomery arithmetic needs an odd modulus > 2")
    if p >= 1 << (32 * L):
        raise UnsafeModulusError(f"{where}: modulus does not fit in {L} limbs")
    if nprime != montgomery_nprime(p):
        raise UnsafeModulusError(
            f"{where}: nprime {nprime:#x} != -p^-1 mod 2^32 = {montgomery_nprime(p):#x}"
        )
    if not cios_bound_holds(p, L):
        raise UnsafeModulusError(
            f"{where}: the device Montgomery routine does not support this modulus. It keeps "
            f"an (L+1)-word accumulator, which is valid only when "
            f"(2p-1) + (p-1)(2^32-1) < 2^(32(L+1))."
        )


def to_limbs(x: int, limbs: int) -> list[int]:
    return [(int(x) >> (32 * i)) & MASK32 for i in range(limbs)]


def from_limbs(words) -> int:
    return sum(int(w) << (32 * i) for i, w in enumerate(words))


@dataclass(frozen=True)
class FieldSpec:
    name: str
    bit_width: int
    limbs: int
    modulus: int
    nprime: int

    def __post_init__(self) -> None:
        if self.limbs not in SUPPORTED_LIMBS:
            raise ValueError(f"limbs must be one of {SUPPORTED_LIMBS}, got {self.limbs}")
        check_montgomery_modulus(self.modulus, self.limbs, self.nprime)

    @property
    def r_mod(self) -> int:
        return (1 << (32 * self.limbs)) % self.modulus

    @property
    def r2_mod(self) -> int:
        return self.r_mod * self.r_mod % self.modulus

    @property
    def r_inv(self) -> int:
        return pow(self.r_mod, -1, self.modulus)

    def to_limbs(self, value: int) -> list[int]:
        return to_limbs(int(value) % self.modulus, self.limbs)

    def montgomery_encode(self, value: int) -> int:
        return (int(value) % self.modulus) * self.r_mod % self.modulus

    def montgomery_decode(self, value: int) -> int:
        return int(value) * self.r_inv % self.modulus

    def montgomery_limbs(self, value: int) -> list[int]:
        return to_limbs(self.montgomery_encode(value), self.limbs)

    def decode_limbs(self, words) -> int:
        """Canonical value of a Montgomery-form limb vector."""
        return self.montgomery_decode(from_limbs(words))


FIELD_SPECS: dict[int, FieldSpec] = {
    32: FieldSpec("p32_2^32_minus_5", 32, 1, 0xFFFFFFFB, 0xCCCCCCCD),
    64: FieldSpec("p64_goldilocks", 64, 2, 0xFFFFFFFF00000001, 0xFFFFFFFF),
    128: FieldSpec("p128_mersenne_2^127_minus_1", 128, 4, (1 << 127) - 1, 0x00000001),
    256: FieldSpec(
        "p255_bls12_381_scalar",
        256,
        8,
        0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001,
        0xFFFFFFFF,
    ),
}


def get_field(bit_width: int) -> FieldSpec:
    try:
        return FIELD_SPECS[int(bit_width)]
    except KeyError as exc:
        supported = ", ".join(str(x) for x in sorted(FIELD_SPECS))
        raise ValueError(
            f"unsupported field bit width {bit_width}; expected one of {supported}"
        ) from exc


def field_for_modulus(q: int, bit_width: int) -> FieldSpec:
    """The field of modulus ``q`` held in ``bit_width / 32`` limbs, guard-checked."""
    bit_width = int(bit_width)
    if bit_width % 32 or bit_width // 32 not in SUPPORTED_LIMBS:
        raise ValueError(f"bit_width must be one of 32, 64, 128, 256, got {bit_width}")
    known = FIELD_SPECS.get(bit_width)
    if known is not None and known.modulus == int(q):
        return known
    if int(q) >= 1 << bit_width:
        raise ValueError(f"q={q} too large for bit_width={bit_width}")
    return FieldSpec(
        name=f"custom_{int(q):#x}",
        bit_width=bit_width,
        limbs=bit_width // 32,
        modulus=int(q),
        nprime=montgomery_nprime(int(q)) if int(q) % 2 else 1,
    )


def stress_value(p: int, limbs: int, rng: random.Random) -> int:
    """One operand in [0, p) drawn to exercise long carry chains and the final subtract."""
    nbits = 32 * limbs
    kind = rng.randrange(8)
    if kind == 0:
        x = p - 1 - rng.randrange(1 << 10)
    elif kind == 1:
        x = p - 1 - rng.getrandbits(rng.randrange(1, nbits + 1))
    elif kind == 2:
        words = (0, 1, MASK32, MASK32 - 1, 0x80000000, 0x7FFFFFFF)
        x = from_limbs([rng.choice(words) for _ in range(limbs)])
    elif kind == 3:
        x = rng.randrange(1 << 10)
    elif kind == 4:
        r = (1 << nbits) % p
        x = rng.choice((r, p - r, r * r % p, 1, p - 1, 0))
    elif kind == 5:
        k = rng.randrange(1, limbs + 1)
        x = ((p >> (32 * k)) << (32 * k)) | rng.getrandbits(32 * k)
    else:
        x = rng.randrange(p)
    return x % p
