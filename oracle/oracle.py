"""CPU oracle for the SumCheck prover path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import
this module. The product (``zkduel_b200``) never does: it has no CPU path.

What is restated here, each from the reference file:line it follows:

* ``sumcheck_reference`` -- the reference's big-integer prover loop
  (``src/zkduel/reference.py:44-110``): g(0), g(1) from evens/odds, g(t>=2) by adding the
  difference repeatedly, fold ``e + r (o - e)`` for rounds ``j < n - 1``.
* ``registry_checksum`` -- the checksum the reference's golden records hold
  (``experiments/h100/tools/validate_vs_registry.py:94-148``): arithmetic-progression
  tables, per round and point ``sum_i (i + 1) limb_i(montgomery(g(t)))``, SHA3 or fixed
  (r = 1) challenges.
* ``sha3_challenge`` -- the Fiat-Shamir rule (``cuda/src/field_sumcheck.cu:857-907``,
  ``benchmarks/field_sweep/triton_sweep.py:474-484``): SHA3-256 over
  ``b"zkduel:field-sweep:v1" || u32le(round) || u32le(each Montgomery limb of g(0..d))``,
  digest read little-endian, reduced mod p.
* ``prove`` -- the full call the prover answers (round polynomials, challenges, final
  claims, checksum). Its challenge at the last round and its final claims extend the
  reference, which derives no last challenge (``field_sumcheck.cu:1057``); they are pinned by
  the verifier identities ``g_j(0) + g_j(1) = g_{j-1}(r_{j-1})`` and
  ``g_{n-1}(r_{n-1}) = expression(f_1(r), ..., f_k(r))``.
* table generators -- ``arith_table`` is the reference's fill
  (``field_sumcheck.cu:123-128,593-611``); ``uniform_table`` / ``bernoulli_table`` are this
  project's seeded generators (counter-based SplitMix64 with rejection to [0, p)), defined
  identically in ``csrc/tables.cuh``.

Parity is pinned: ``tests/golden/`` holds the reference's registry checksums and outputs of
the reference's own ``sumcheck_reference`` on seeded tables, and ``tests/test_oracle.py``
checks this module against both.
"""

from __future__ import annotations

import hashlib
from typing import Iterable, Mapping, Sequence

import numpy as np

DOMAIN = b"zkduel:field-sweep:v1"
MASK32 = 0xFFFFFFFF
MASK64 = (1 << 64) - 1


# --------------------------------------------------------------------------------------
# expressions (same normal form as the reference's _expr.py:27-67)
# --------------------------------------------------------------------------------------


def _normalize(expression) -> list[tuple[int, tuple[str, ...]]]:
    out = []
    for term in expression:
        if (
            isinstance(term, (list, tuple))
            and len(term) == 2
            and not isinstance(term[0], str)
            and not isinstance(term[1], str)
            and isinstance(term[0], int)
        ):
            out.append((int(term[0]), tuple(term[1])))
        else:
            out.append((1, tuple(term)))
    return out


def _vars(expression) -> list[str]:
    seen: list[str] = []
    for _c, names in _normalize(expression):
        for v in names:
            if v not in seen:
                seen.append(v)
    return seen


def indexed_terms(expression, order: Sequence[str] | None = None):
    """Terms as ``(coeff, [table index])`` with tables numbered by ``order``."""
    names = list(order) if order is not None else _vars(expression)
    pos = {v: i for i, v in enumerate(names)}
    return [(c, [pos[v] for v in f]) for c, f in _normalize(expression)], len(names)


# --------------------------------------------------------------------------------------
# reference.py restated
# --------------------------------------------------------------------------------------


def sumcheck_reference(
    eval_tables: Mapping[str, Iterable[int] | np.ndarray],
    *,
    q: int,
    expression,
    challenges: Sequence[int],
    num_rounds: int,
) -> tuple[int, np.ndarray]:
    """``(claim0, evals[num_rounds][degree + 1])`` -- reference.py:44-110."""
    terms, k = indexed_terms(expression)
    names = _vars(expression)
    degree = max(len(f) for _c, f in terms)
    tabs = [[int(x) % q for x in np.asarray(eval_tables[v], dtype=object).reshape(-1)] for v in names]
    size = 1 << num_rounds
    for v, t in zip(names, tabs):
        if len(t) != size:
            raise ValueError(f"Table for {v!r} has length {len(t)}, expected {size}")

    def compose_sum(cols) -> int:
        total = 0
        for i in range(len(cols[0])):
            for c, f in terms:
                prod = c % q
                for x in f:
                    prod = prod * cols[x][i] % q
                total += prod
        return total % q

    claim0 = compose_sum(tabs)
    evals = []
    for rnd in range(num_rounds):
        ev = [t[0::2] for t in tabs]
        od = [t[1::2] for t in tabs]
        df = [[(o - e) % q for e, o in zip(a, b)] for a, b in zip(ev, od)]
        g = [compose_sum(ev), compose_sum(od)]
        cur = [list(x) for x in od]
        for _t in range(2, degree + 1):
            cur = [[(c + d) % q for c, d in zip(a, b)] for a, b in zip(cur, df)]
            g.append(compose_sum(cur))
        evals.append(g)
        if rnd < num_rounds - 1:
            r = int(challenges[rnd]) % q
            tabs = [[(e + r * d) % q for e, d in zip(a, b)] for a, b in zip(ev, df)]
    return claim0, np.array(evals, dtype=object)


# --------------------------------------------------------------------------------------
# transcript, checksum, interpolation
# --------------------------------------------------------------------------------------


def mont_limbs(x: int, p: int, limbs: int) -> list[int]:
    m = (int(x) % p) * ((1 << (32 * limbs)) % p) % p
    return [(m >> (32 * i)) & MASK32 for i in range(limbs)]


def sha3_challenge(round_idx: int, point_values: Sequence[int], p: int, limbs: int) -> int:
    h = hashlib.sha3_256()
    h.update(DOMAIN)
    h.update(int(round_idx).to_bytes(4, "little"))
    for v in point_values:
        for w in mont_limbs(v, p, limbs):
            h.update(w.to_bytes(4, "little"))
    return int.from_bytes(h.digest(), "little") % p


def round_checksum(point_values: Sequence[int], p: int, limbs: int) -> int:
    return sum(sum((i + 1) * w for i, w in enumerate(mont_limbs(v, p, limbs))) for v in point_values)


def lagrange_eval(values: Sequence[int], r: int, p: int) -> int:
    """Value at r of the polynomial through (t, values[t]), t = 0..d."""
    d1 = len(values)
    total = 0
    for t in range(d1):
        num, den = 1, 1
        for s in range(d1):
            if s != t:
                num = num * (r - s) % p
                den = den * (t - s) % p
        total += values[t] * num * pow(den, -1, p)
    return total % p


# --------------------------------------------------------------------------------------
# the prover call
# --------------------------------------------------------------------------------------


def prove(
    terms,
    num_tables: int,
    p: int,
    limbs: int,
    tables: Sequence[Sequence[int]],
    challenge_mode: str = "sha3",
    explicit: Sequence[int] | None = None,
) -> dict:
    """Round polynomials, challenges, final claims and checksum of one proof.

    ``terms``: ``[(coeff, [table index, ...]), ...]``; ``tables``: canonical values,
    ``num_tables`` lists of length 2^n. Challenge modes: ``sha3`` (derived from the
    transcript), ``fixed`` (r = 1) or ``explicit`` (``explicit[j]``).
    """
    tabs = [[int(x) % p for x in t] for t in tables]
    assert len(tabs) == num_tables
    size = len(tabs[0])
    n = size.bit_length() - 1
    assert size == 1 << n and n >= 1
    degree = max(len(f) for _c, f in terms)
    checksum = 0
    polys, chals = [], []
    for rnd in range(n):
        half = len(tabs[0]) // 2
        ev = [t[0::2] for t in tabs]
        df = [[(t[2 * i + 1] - t[2 * i]) % p for i in range(half)] for t in tabs]
        g = []
        cur = [list(e) for e in ev]
        for t in range(degree + 1):
            if t:
                cur = [[(c + d) % p for c, d in zip(a, b)] for a, b in zip(cur, df)]
            total = 0
            for i in range(half):
                for c, f in terms:
                    prod = c % p
                    for x in f:
                        prod = prod * cur[x][i] % p
                    total += prod
            g.append(total % p)
        polys.append(g)
        checksum += round_checksum(g, p, limbs)
        if challenge_mode == "sha3":
            r = sha3_challenge(rnd, g, p, limbs)
        elif challenge_mode == "fixed":
            r = 1
        elif challenge_mode == "explicit":
            r = int(explicit[rnd]) % p
        else:
            raise ValueError(challenge_mode)
        chals.append(r)
        tabs = [[(e + r * d) % p for e, d in zip(a, b)] for a, b in zip(ev, df)]
    final_vals = [t[0] for t in tabs]
    return {
        "round_polys": polys,
        "challenges": chals,
        "claim0": (polys[0][0] + polys[0][1]) % p,
        "final_claim": lagrange_eval(polys[-1], chals[-1], p),
        "final_values": final_vals,
        "checksum": checksum,
    }


def evaluate_terms(terms, values: Sequence[int], p: int) -> int:
    total = 0
    for c, f in terms:
        prod = c % p
        for x in f:
            prod = prod * values[x] % p
        total += prod
    return total % p


def registry_checksum(terms, num_tables: int, p: int, limbs: int, rounds: int, seed: int,
                      challenge_mode: str) -> int:
    """Checksum of one run on the reference's arithmetic-progression tables
    (validate_vs_registry.py:94-148); the golden records hold twice this value."""
    tables = [arith_table(seed, v, 1 << rounds, p) for v in range(num_tables)]
    return prove(terms, num_tables, p, limbs, tables, challenge_mode)["checksum"]


# --------------------------------------------------------------------------------------
# table generators (identical definitions in csrc/tables.cu)
# --------------------------------------------------------------------------------------


def arith_table(seed: int, var: int, size: int, p: int) -> list[int]:
    """field_sumcheck.cu:123-128: (seed + 7919 (var + 1) + 104729 (off + 1)) mod p."""
    base = (seed & MASK32) + 7919 * (var + 1)
    return [(base + 104729 * (off + 1)) % p for off in range(size)]


_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
MAX_ATTEMPTS = 64


def _mix64(z: np.ndarray) -> np.ndarray:
    z = np.array(z, dtype=np.uint64, copy=True)
    with np.errstate(over="ignore"):
        z ^= z >> np.uint64(30)
        z *= _M1
        z ^= z >> np.uint64(27)
        z *= _M2
        z ^= z >> np.uint64(31)
    return z


def splitmix64(x) -> np.ndarray:
    with np.errstate(over="ignore"):
        return _mix64(np.asarray(x, dtype=np.uint64) + _G)


def table_key(seed: int, table: int) -> np.uint64:
    with np.errstate(over="ignore"):
        inner = splitmix64(np.uint64((table + 0x632BE59BD9B4E019) & MASK64))
        return splitmix64(np.uint64(seed & MASK64) ^ inner)[()]


def _words(key: np.uint64, idx: np.ndarray, attempt: int, limbs: int) -> list[np.ndarray]:
    """The ``limbs`` 32-bit words of draw ``attempt`` for elements ``idx``."""
    out = []
    with np.errstate(over="ignore"):
        for w in range((limbs + 1) // 2):
            ctr = (idx << np.uint64(8)) | np.uint64((attempt << 2) | w)
            z = splitmix64(key + ctr)
            out.append(z & np.uint64(MASK32))
            out.append(z >> np.uint64(32))
    return out[:limbs]


def uniform_table(seed: int, table: int, size: int, p: int, limbs: int) -> list[int]:
    """Uniform in [0, p): draw 32 L bits, keep the low bit_length(p) bits, reject >= p."""
    key = table_key(seed, table)
    idx = np.arange(size, dtype=np.uint64)
    bits = p.bit_length()
    out = [None] * size
    pending = np.arange(size)
    for attempt in range(MAX_ATTEMPTS):
        if pending.size == 0:
            break
        ws = _words(key, idx[pending], attempt, limbs)
        keep = []
        for j, e in enumerate(pending.tolist()):
            x = 0
            for i, w in enumerate(ws):
                x |= int(w[j]) << (32 * i)
            x &= (1 << bits) - 1
            if x < p:
                out[e] = x
            else:
                keep.append(e)
        pending = np.array(keep, dtype=np.int64)
    for e in pending.tolist():  # never reached in practice: the last draw, masked, minus p
        ws = _words(key, idx[[e]], MAX_ATTEMPTS - 1, limbs)
        x = sum(int(w[0]) << (32 * i) for i, w in enumerate(ws)) & ((1 << bits) - 1)
        out[e] = x - p
    return out


def bernoulli_table(seed: int, table: int, size: int) -> list[int]:
    """0/1 selectors: the low bit of the element's first draw."""
    key = table_key(seed, table)
    idx = np.arange(size, dtype=np.uint64)
    w = _words(key, idx, 0, 1)[0]
    return [int(x) & 1 for x in w]


def make_tables(kinds: Sequence[str], seed: int, size: int, p: int, limbs: int,
                arith_index: Sequence[int] | None = None) -> list[list[int]]:
    """One table per entry of ``kinds`` ("uniform", "bernoulli", "arith")."""
    out = []
    for k, kind in enumerate(kinds):
        if kind == "uniform":
            out.append(uniform_table(seed, k, size, p, limbs))
        elif kind == "bernoulli":
            out.append(bernoulli_table(seed, k, size))
        elif kind == "arith":
            v = arith_index[k] if arith_index is not None else k
            out.append(arith_table(seed, v, size, p))
        else:
            raise ValueError(kind)
    return out
