"""Seeded proof streams: the mixed batch and the served request stream.

batched   ``count`` (512) independent proofs; num_vars uniform in {10..20}; field 64- or
          256-bit by coin flip; each expression a sum of 1-3 products of 2-6 distinct tables
          drawn from 2-8 tables (degree 2-6); tables uniform in [0, p); per-proof seeds from
          one master seed.
served    a Poisson arrival stream over the 2^127 - 1 field: num_vars log-uniform in
          [12, 24], sum-of-products expressions of degree 3-7 over up to 8 tables, arrival
          rate chosen from a measured service time (``rate`` is an argument).

Tables are named t0..t{k-1}; only tables that some term uses are inputs of the proof.
"""

from __future__ import annotations

import math
import random
from dataclasses import dataclass

from .expression import encode_expression, expression_vars


@dataclass(frozen=True)
class ProofSpec:
    index: int
    bit_width: int
    num_vars: int
    seed: int
    expression: tuple  # ((coeff, (names...)), ...)

    @property
    def var_names(self) -> list[str]:
        return expression_vars(self.expression)

    @property
    def num_tables(self) -> int:
        return len(self.var_names)

    @property
    def degree(self) -> int:
        return max(len(f) for _c, f in self.expression)

    def encoded(self):
        return encode_expression(self.expression)


def _random_expression(rng: random.Random, max_tables: int, min_deg: int, max_deg: int,
                       max_terms: int) -> tuple:
    k = rng.randint(2, max_tables)
    terms = []
    for _ in range(rng.randint(1, max_terms)):
        size = rng.randint(min(min_deg, k), min(max_deg, k))
        names = rng.sample([f"t{i}" for i in range(k)], size)
        terms.append((1, tuple(names)))
    return tuple(terms)


def batched_stream(count: int = 512, seed: int = 0) -> list[ProofSpec]:
    rng = random.Random(seed)
    out = []
    for i in range(count):
        n = rng.randint(10, 20)
        bw = 64 if rng.random() < 0.5 else 256
        expr = _random_expression(rng, 8, 2, 6, 3)
        out.append(ProofSpec(i, bw, n, rng.getrandbits(63), expr))
    return out


@dataclass(frozen=True)
class Request:
    spec: ProofSpec
    arrival_s: float


def served_stream(count: int = 20000, rate_per_s: float = 1000.0, seed: int = 1,
                  min_vars: int = 12, max_vars: int = 24) -> list[Request]:
    """Poisson arrivals (exponential gaps at ``rate_per_s``) of 128-bit proofs."""
    rng = random.Random(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.expovariate(rate_per_s)
        n = int(round(math.exp(rng.uniform(math.log(min_vars), math.log(max_vars)))))
        n = max(min_vars, min(max_vars, n))
        expr = _random_expression(rng, 8, 3, 7, 3)
        # degree 3-7 needs one term at least that long: lengthen the first if needed
        if max(len(f) for _c, f in expr) < 3:
            expr = ((1, tuple(f"t{j}" for j in range(3))),) + expr[1:]
        out.append(Request(ProofSpec(i, 128, n, rng.getrandbits(63), expr), t))
    return out
