"""The named proving workloads: the plain single-proof shapes and their table kinds.

plain_p32         poly_ab over p = 2^32 - 5, n = 16, both tables uniform (seed 0).
plain_goldilocks  vanilla_zerocheck_hp (eq(r, x) (qM a b + qL a + qR b - qO c + qC)) over
                  Goldilocks, n = 24: a, b, c, eq (w1, w2, w3, fz1) and qC uniform; the
                  selectors qM, qL, qR, qO Bernoulli(1/2).
plain_bls         poly_abcg_plus_deg (a b c g + d e g) over the BLS12-381 scalar field,
                  n = 22, all tables uniform.
"""

from __future__ import annotations

from dataclasses import dataclass

from .expression import expression_vars
from .workloads import WORKLOADS


@dataclass(frozen=True)
class PlainConfig:
    name: str
    workload: str
    bit_width: int
    num_vars: int
    bernoulli: tuple[str, ...] = ()
    seed: int = 0

    @property
    def expression(self):
        return WORKLOADS[self.workload]

    def table_kinds(self) -> list[str]:
        return ["bernoulli" if v in self.bernoulli else "uniform" for v in expression_vars(self.expression)]

    def with_vars(self, n: int) -> "PlainConfig":
        return PlainConfig(self.name, self.workload, self.bit_width, n, self.bernoulli, self.seed)


PLAIN_CONFIGS = {
    "plain_p32": PlainConfig("plain_p32", "poly_ab", 32, 16),
    "plain_goldilocks": PlainConfig("plain_goldilocks", "vanilla_zerocheck_hp", 64, 24, ("qM", "qL", "qR", "qO")),
    "plain_bls": PlainConfig("plain_bls", "poly_abcg_plus_deg", 256, 22),
}
