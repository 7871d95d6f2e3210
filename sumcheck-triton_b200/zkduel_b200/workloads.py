"""Constraint-expression registry.

``WORKLOADS`` holds the same expressions, under the same names and aliases, as the
reference's registry (``src/zkduel/workloads.py:11-255``): the seven diagnostic
polynomials, the 25 zkPHIRE constraints and their ``zkphire_N`` aliases, with
``alpha = 7`` in the permutation checks. The expressions are the interface of the prover
(callers name them), so they are kept term for term.

``KERNEL_WORKLOADS`` lists the 32 workloads of the reference's CUDA executable
(``cuda/src/field_sumcheck.cu:696-733``) with their numeric id and the order in which that
executable numbers their tables (``benchmarks/field_sweep/workload_specs.py``). The table
order matters for one thing only: the reference fills table ``v`` with
``seed + 7919 (v + 1) + 104729 (off + 1)``, so reproducing its checksums needs the same
numbering.
"""

from __future__ import annotations

from dataclasses import dataclass

from .expression import Expression, expression_degree, expression_vars

alpha = 7

WORKLOADS: dict[str, Expression] = {
    "poly_a": [["a"]],
    "poly_ab": [["a", "b"]],
    "poly_ab_plus_c": [["a", "b"], ["c"]],
    "poly_abc": [["a", "b", "c"]],
    "poly_aabbc": [["a", "a", "b", "b", "c"]],
    "poly_abc_plus_de": [["a", "b", "c"], ["d", "e"]],
    "poly_abcg_plus_deg": [["a", "b", "c", "g"], ["d", "e", "g"]],
    "linear": [["a"]],
    "quadratic": [["a", "b"]],
    "cubic_plus_quad": [["a", "b", "c"], ["d", "e"]],
    "opencheck": [["y1", "k1"], ["y2", "k2"], ["y3", "k3"], ["y4", "k4"], ["y5", "k5"], ["y6", "k6"]],
    "vanilla_zerocheck_hp": [
        ["qL", "w1", "fz1"],
        ["qR", "w2", "fz1"],
        ["qM", "w1", "w2", "fz1"],
        (-1, ["qO", "w3", "fz1"]),
        ["qC", "fz1"],
    ],
    "vanilla_permcheck_hp": [
        ["pi", "fz2"],
        (-1, ["p1", "p2", "fz2"]),
        (alpha, ["phi", "D1", "D2", "D3", "fz2"]),
        (-alpha, ["N1", "N2", "N3", "fz2"]),
    ],
    "jellyfish_zerocheck_hp": [
        ["qL", "w1", "fz"],
        ["qR", "w2", "fz"],
        ["qM", "w1", "w2", "fz"],
        (-1, ["qO", "w3", "fz"]),
        ["q1", "w1", "fz"],
        ["q2", "w2", "fz"],
        ["q3", "w3", "fz"],
        ["q4", "w4", "fz"],
        (-1, ["qO", "w5", "fz"]),
        ["qM1", "w1", "w2", "fz"],
        ["qM2", "w3", "w4", "fz"],
        ["qH1", "w1", "w1", "w1", "w1", "w1", "fz"],
        ["qH2", "w2", "w2", "w2", "w2", "w2", "fz"],
        ["qH3", "w3", "w3", "w3", "w3", "w3", "fz"],
        ["qH4", "w4", "w4", "w4", "w4", "w4", "fz"],
        ["qECC", "w1", "w2", "w3", "w4", "fz"],
        ["qc", "fz"],
    ],
    "jellyfish_permcheck_hp": [
        ["pi", "fz"],
        (-1, ["p1", "p2", "fz"]),
        (alpha, ["phi", "D1", "D2", "D3", "D4", "D5", "fz"]),
        (-alpha, ["N1", "N2", "N3", "N4", "N5", "fz"]),
    ],
    "verifiable_asics": [["qadd", "a"], ["qadd", "b"], ["qmul", "a", "b"]],
    "spartan_1": [["A", "B", "fz"], (-1, ["C", "fz"])],
    "spartan_2": [["ABC", "Z"]],
    "witness_non_id_point": [
        ["q_non-id-point", "y", "y"],
        (-1, ["q_non-id-point", "x", "x", "x"]),
        (-5, ["q_non-id-point"]),
    ],
    "witness_id_point_1": [
        ["q_point", "x", "y", "y"],
        (-1, ["q_point", "x", "x", "x", "x"]),
        (-5, ["q_point", "x"]),
    ],
    "witness_id_point_2": [
        ["q_point", "y", "y", "y"],
        (-1, ["q_point", "y", "x", "x", "x"]),
        (-5, ["q_point", "y"]),
    ],
    "incomplete_addition_1": [
        ["q_add-incomplete", "x_r", "x_p", "x_p"],
        (-2, ["q_add-incomplete", "x_r", "x_p", "x_q"]),
        ["q_add-incomplete", "x_r", "x_q", "x_q"],
        ["q_add-incomplete", "x_q", "x_p", "x_p"],
        (-2, ["q_add-incomplete", "x_q", "x_q", "x_p"]),
        ["q_add-incomplete", "x_q", "x_q", "x_q"],
        ["q_add-incomplete", "x_p", "x_p", "x_p"],
        (-2, ["q_add-incomplete", "x_p", "x_p", "x_q"]),
        ["q_add-incomplete", "x_p", "x_q", "x_q"],
        (-1, ["q_add-incomplete", "y_p", "y_p"]),
        (2, ["q_add-incomplete", "y_p", "y_q"]),
        (-1, ["q_add-incomplete", "y_q", "y_q"]),
    ],
    "incomplete_addition_2": [
        ["q_add-incomplete", "y_r", "x_p"],
        (-1, ["q_add-incomplete", "y_r", "x_q"]),
        ["q_add-incomplete", "y_q", "x_p"],
        (-1, ["q_add-incomplete", "y_q", "x_q"]),
        (-1, ["q_add-incomplete", "y_p", "x_q"]),
        ["q_add-incomplete", "y_p", "x_r"],
        (-1, ["q_add-incomplete", "y_q", "x_r"]),
        ["q_add-incomplete", "y_q", "x_q"],
    ],
    "complete_addition_1": [
        ["q_add", "x_q", "x_q", "lambda"],
        (-2, ["q_add", "x_q", "x_p", "lambda"]),
        ["q_add", "x_p", "x_p", "lambda"],
        (-1, ["q_add", "x_q", "y_q"]),
        ["q_add", "x_q", "y_p"],
        ["q_add", "x_p", "y_q"],
        (-1, ["q_add", "x_p", "y_p"]),
    ],
    "complete_addition_2": [
        (2, ["q_add", "y_p", "lambda"]),
        (-3, ["q_add", "x_p", "x_p"]),
        (-2, ["q_add", "x_q", "y_p", "lambda", "alpha"]),
        (3, ["q_add", "x_q", "x_p", "x_p", "alpha"]),
        (2, ["q_add", "x_p", "y_p", "lambda", "alpha"]),
        (-3, ["q_add", "x_p", "x_p", "x_p", "alpha"]),
    ],
    "complete_addition_3": [
        ["q_add", "x_p", "x_q", "x_q", "lambda", "lambda"],
        (-1, ["q_add", "x_p", "x_q", "x_q", "x_q"]),
        (-1, ["q_add", "x_p", "x_q", "x_q", "x_r"]),
        (-1, ["q_add", "x_p", "x_p", "x_q", "x_q"]),
        (-1, ["q_add", "x_p", "x_p", "x_q", "lambda", "lambda"]),
        ["q_add", "x_p", "x_p", "x_p", "x_q"],
        ["q_add", "x_p", "x_p", "x_q", "x_r"],
        ["q_add", "x_p", "x_p", "x_q", "x_q"],
    ],
    "complete_addition_4": [
        ["q_add", "x_p", "x_p", "x_q", "x_q", "lambda"],
        (-1, ["q_add", "x_p", "x_q", "x_q", "x_r", "lambda"]),
        (-1, ["q_add", "x_p", "x_q", "x_q", "y_p"]),
        (-1, ["q_add", "x_p", "x_q", "x_q", "y_r"]),
        (-1, ["q_add", "x_p", "x_p", "x_p", "x_q", "lambda"]),
        ["q_add", "x_p", "x_p", "x_q", "x_r", "lambda"],
        ["q_add", "x_p", "x_p", "x_q", "y_p"],
        ["q_add", "x_p", "x_p", "x_q", "y_r"],
    ],
    "complete_addition_5": [
        ["q_add", "x_p", "x_q", "y_q", "lambda", "lambda"],
        ["q_add", "x_p", "x_q", "y_p", "lambda", "lambda"],
        (-1, ["q_add", "x_p", "x_p", "x_q", "y_q"]),
        (-1, ["q_add", "x_p", "x_p", "x_q", "y_p"]),
        (-1, ["q_add", "x_p", "x_q", "x_q", "y_q"]),
        (-1, ["q_add", "x_p", "x_q", "x_q", "y_p"]),
        (-1, ["q_add", "x_p", "x_q", "y_q", "x_r"]),
        (-1, ["q_add", "x_p", "x_q", "y_p", "x_r"]),
    ],
    "complete_addition_6": [
        ["q_add", "x_p", "x_p", "x_q", "y_q", "lambda"],
        ["q_add", "x_p", "x_p", "x_q", "y_p", "lambda"],
        (-1, ["q_add", "x_p", "x_q", "y_p", "x_r", "lambda"]),
        (-1, ["q_add", "x_p", "x_q", "y_q", "x_r", "lambda"]),
        (-1, ["q_add", "x_p", "x_q", "y_p", "y_p"]),
        (-1, ["q_add", "x_p", "x_q", "y_p", "y_q"]),
        (-1, ["q_add", "x_p", "x_q", "y_p", "y_r"]),
        (-1, ["q_add", "x_p", "x_q", "y_q", "y_r"]),
    ],
    "complete_addition_7": [
        ["q_add", "x_r"],
        (-1, ["q_add", "x_q"]),
        (-1, ["q_add", "x_p", "x_r", "beta"]),
        ["q_add", "x_p", "x_q", "beta"],
    ],
    "complete_addition_8": [
        ["q_add", "y_r"],
        (-1, ["q_add", "y_q"]),
        (-1, ["q_add", "x_p", "y_r", "beta"]),
        ["q_add", "x_p", "y_q", "beta"],
    ],
    "complete_addition_9": [
        ["q_add", "x_r"],
        (-1, ["q_add", "x_p"]),
        (-1, ["q_add", "x_q", "x_r", "gamma"]),
        ["q_add", "x_p", "x_q", "gamma"],
    ],
    "complete_addition_10": [
        ["q_add", "y_r"],
        (-1, ["q_add", "y_p"]),
        (-1, ["q_add", "x_q", "y_r", "gamma"]),
        ["q_add", "x_q", "y_p", "gamma"],
    ],
    "complete_addition_11": [
        ["q_add", "x_r"],
        (-1, ["q_add", "x_q", "x_r", "alpha"]),
        ["q_add", "x_p", "x_r", "alpha"],
        (-1, ["q_add", "y_q", "x_r", "delta"]),
        (-1, ["q_add", "y_p", "x_r", "delta"]),
    ],
    "complete_addition_12": [
        ["q_add", "y_r"],
        (-1, ["q_add", "x_q", "y_r", "alpha"]),
        ["q_add", "x_p", "y_r", "alpha"],
        (-1, ["q_add", "y_q", "y_r", "delta"]),
        (-1, ["q_add", "y_p", "y_r", "delta"]),
    ],
}

_ALIASES = {
    "a": "poly_a",
    "ab": "poly_ab",
    "ab_plus_c": "poly_ab_plus_c",
    "abc": "poly_abc",
    "aabbc": "poly_aabbc",
    "abc_plus_de": "poly_abc_plus_de",
    "abcg_plus_deg": "poly_abcg_plus_deg",
    "zkphire_0": "verifiable_asics",
    "zkphire_1": "spartan_1",
    "zkphire_2": "spartan_2",
    "zkphire_3": "witness_non_id_point",
    "zkphire_4": "witness_id_point_1",
    "zkphire_5": "witness_id_point_2",
    "zkphire_6": "incomplete_addition_1",
    "zkphire_7": "incomplete_addition_2",
    **{f"zkphire_{8 + i}": f"complete_addition_{1 + i}" for i in range(12)},
    "zkphire_20": "vanilla_zerocheck_hp",
    "zkphire_21": "vanilla_permcheck_hp",
    "zkphire_22": "jellyfish_zerocheck_hp",
    "zkphire_23": "jellyfish_permcheck_hp",
    "zkphire_24": "opencheck",
    "hyperplonk_zero": "vanilla_zerocheck_hp",
    "hyperplonk_perm": "vanilla_permcheck_hp",
    "hyperplonk_open": "opencheck",
}
for _alias, _target in _ALIASES.items():
    WORKLOADS[_alias] = WORKLOADS[_target]


def get_workload(name: str) -> Expression:
    try:
        return WORKLOADS[name]
    except KeyError as exc:
        known = ", ".join(sorted(WORKLOADS))
        raise KeyError(f"unknown workload {name!r}; known: {known}") from exc


@dataclass(frozen=True)
class KernelWorkload:
    """One workload of the reference CUDA executable: id, name, registry name, table order."""

    ident: int
    name: str
    registry_name: str
    table_order: tuple[str, ...]

    @property
    def expression(self) -> Expression:
        return WORKLOADS[self.registry_name]

    @property
    def degree(self) -> int:
        return expression_degree(self.expression)

    @property
    def num_vars(self) -> int:
        return len(self.table_order)

    def table_index(self) -> list[int]:
        """Kernel table index of each registry variable, in ``expression_vars`` order."""
        pos = {v: i for i, v in enumerate(self.table_order)}
        return [pos[v] for v in expression_vars(self.expression)]


def _kw(ident, name, reg, order):
    return KernelWorkload(ident, name, reg, tuple(order.split()))


KERNEL_WORKLOADS: tuple[KernelWorkload, ...] = (
    _kw(1, "poly_a", "poly_a", "a"),
    _kw(2, "poly_ab", "poly_ab", "a b"),
    _kw(3, "poly_ab_plus_c", "poly_ab_plus_c", "a b c"),
    _kw(4, "poly_abc", "poly_abc", "a b c"),
    _kw(5, "poly_aabbc", "poly_aabbc", "a b c"),
    _kw(6, "poly_abc_plus_de", "poly_abc_plus_de", "a b c d e"),
    _kw(7, "poly_abcg_plus_deg", "poly_abcg_plus_deg", "a b c g d e"),
    _kw(8, "zk_verifiable_asics", "zkphire_0", "qadd a b qmul"),
    _kw(9, "zk_spartan_1", "zkphire_1", "A B fz C"),
    _kw(10, "zk_spartan_2", "zkphire_2", "ABC Z"),
    _kw(11, "zk_witness_non_id", "zkphire_3", "q_non-id-point y x"),
    _kw(12, "zk_complete_add_1", "zkphire_8", "q_add x_q x_p lambda y_q y_p"),
    _kw(13, "zk_complete_add_7", "zkphire_14", "q_add x_r x_q x_p beta"),
    _kw(14, "zk_complete_add_8", "zkphire_15", "q_add y_r y_q x_p beta"),
    _kw(15, "zk_witness_id_point_1", "zkphire_4", "q_point x y"),
    _kw(16, "zk_witness_id_point_2", "zkphire_5", "q_point y x"),
    _kw(17, "zk_incomplete_add_1", "zkphire_6", "q_add-incomplete x_r x_p x_q y_p y_q"),
    _kw(18, "zk_incomplete_add_2", "zkphire_7", "q_add-incomplete y_r x_p x_q y_q y_p x_r"),
    _kw(19, "zk_complete_add_2", "zkphire_9", "q_add y_p lambda x_p x_q alpha"),
    _kw(20, "zk_complete_add_3", "zkphire_10", "q_add x_p x_q lambda x_r"),
    _kw(21, "zk_complete_add_4", "zkphire_11", "q_add x_p x_q lambda x_r y_p y_r"),
    _kw(22, "zk_complete_add_5", "zkphire_12", "q_add x_p x_q y_q lambda y_p x_r"),
    _kw(23, "zk_complete_add_6", "zkphire_13", "q_add x_p x_q y_q lambda y_p x_r y_r"),
    _kw(24, "zk_complete_add_9", "zkphire_16", "q_add x_r x_p x_q gamma"),
    _kw(25, "zk_complete_add_10", "zkphire_17", "q_add y_r y_p x_q gamma"),
    _kw(26, "zk_complete_add_11", "zkphire_18", "q_add x_r x_q alpha x_p y_q delta y_p"),
    _kw(27, "zk_complete_add_12", "zkphire_19", "q_add y_r x_q alpha x_p y_q delta y_p"),
    _kw(28, "zk_vanilla_zerocheck_hp", "zkphire_20", "qL w1 fz1 qR w2 qM qO w3 qC"),
    _kw(29, "zk_vanilla_permcheck_hp", "zkphire_21", "pi fz2 p1 p2 phi D1 D2 D3 N1 N2 N3"),
    _kw(
        30,
        "zk_jellyfish_zerocheck_hp",
        "zkphire_22",
        "qL w1 fz qR w2 qM qO w3 q1 q2 q3 q4 w4 w5 qM1 qM2 qH1 qH2 qH3 qH4 qECC qc",
    ),
    _kw(
        31,
        "zk_jellyfish_permcheck_hp",
        "zkphire_23",
        "pi fz p1 p2 phi D1 D2 D3 D4 D5 N1 N2 N3 N4 N5",
    ),
    _kw(32, "zk_opencheck", "zkphire_24", "y1 k1 y2 k2 y3 k3 y4 k4 y5 k5 y6 k6"),
)
KERNEL_WORKLOAD_BY_NAME = {w.name: w for w in KERNEL_WORKLOADS}
# zkphire ids follow the registry aliases, not the kernel id order
KERNEL_ALIASES = {
    alias: next(w.name for w in KERNEL_WORKLOADS if w.registry_name == alias)
    for alias in (f"zkphire_{i}" for i in range(25))
}


def get_kernel_workload(name: str) -> KernelWorkload:
    name = KERNEL_ALIASES.get(name, name)
    try:
        return KERNEL_WORKLOAD_BY_NAME[name]
    except KeyError as exc:
        known = ", ".join(sorted([*KERNEL_WORKLOAD_BY_NAME, *KERNEL_ALIASES]))
        raise KeyError(f"unknown kernel workload {name!r}; known: {known}") from exc
