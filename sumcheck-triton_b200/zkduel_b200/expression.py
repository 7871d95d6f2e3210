"""Constraint expressions: parsing, normal form and the flat encoding the device reads.

An expression is a sum of products of table names. Two spellings are accepted, as in the
reference (``src/zkduel/_expr.py:27-54``):

* ``[["a", "b"], ["c"]]`` -- every term has coefficient 1;
* ``[(3, ["a", "b"]), (-1, ["c"])]`` -- ``(coefficient, factors)`` pairs.

Variables are numbered in first-seen order (``_expr.py:57-63``); that order is the order of
the tables the prover takes. The degree is the longest term (``_expr.py:66-67``).
Errors match the reference: ``TypeError`` for malformed terms, ``ValueError`` for an empty
expression.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Sequence

Expression = Sequence[Any]
NormalTerm = tuple[int, tuple[str, ...]]


def _coeff_pair(term: Any) -> tuple[int, tuple[str, ...]] | None:
    """``(c, factors)`` if ``term`` is a coefficient pair, else None."""
    if not isinstance(term, (list, tuple)) or len(term) != 2:
        return None
    coeff, factors = term
    if isinstance(coeff, str) or isinstance(factors, str):
        return None
    try:
        c = int(coeff)
    except (TypeError, ValueError):
        return None
    try:
        names = tuple(factors)
    except TypeError:
        return None
    if not all(isinstance(v, str) for v in names):
        return None
    return c, names


def normalize_expression(expression: Expression) -> tuple[NormalTerm, ...]:
    out: list[NormalTerm] = []
    for term in expression:
        pair = _coeff_pair(term)
        if pair is not None:
            out.append(pair)
            continue
        if isinstance(term, str):
            raise TypeError("Expression terms must be sequences of variable names")
        try:
            names = tuple(term)
        except TypeError as exc:
            raise TypeError("Expression terms must be sequences") from exc
        if not all(isinstance(v, str) for v in names):
            raise TypeError(
                "Expression terms must contain variable names, or be "
                "(coefficient, variable_names) pairs"
            )
        out.append((1, names))
    if not out:
        raise ValueError("expression must contain at least one term")
    return tuple(out)


def expression_vars(expression: Expression) -> list[str]:
    order: dict[str, None] = {}
    for _c, names in normalize_expression(expression):
        for v in names:
            order.setdefault(v, None)
    return list(order)


def expression_degree(expression: Expression) -> int:
    return max(len(names) for _c, names in normalize_expression(expression))


@dataclass(frozen=True)
class EncodedExpression:
    """Flat form handed to the C ABI (``sc_expr_compile``).

    ``flat[term_offsets[i] : term_offsets[i] + term_lens[i]]`` are the table indices of
    term ``i``; ``coeffs[i]`` its integer coefficient (reduced mod p on the device side).
    """

    var_names: tuple[str, ...]
    coeffs: tuple[int, ...]
    term_lens: tuple[int, ...]
    term_offsets: tuple[int, ...]
    flat: tuple[int, ...]

    @property
    def num_vars(self) -> int:
        return len(self.var_names)

    @property
    def num_terms(self) -> int:
        return len(self.coeffs)

    @property
    def degree(self) -> int:
        return max(self.term_lens)


def encode_expression(expression: Expression) -> EncodedExpression:
    terms = normalize_expression(expression)
    names = expression_vars(expression)
    index = {v: i for i, v in enumerate(names)}
    coeffs, lens, offsets, flat = [], [], [], []
    for c, factors in terms:
        offsets.append(len(flat))
        coeffs.append(int(c))
        lens.append(len(factors))
        flat.extend(index[v] for v in factors)
    return EncodedExpression(tuple(names), tuple(coeffs), tuple(lens), tuple(offsets), tuple(flat))


def evaluate(expression: Expression, values: dict[str, int], q: int) -> int:
    """Host evaluation of the expression at one point (used for the verifier identity)."""
    total = 0
    for c, names in normalize_expression(expression):
        prod = c % q
        for v in names:
            prod = prod * values[v] % q
        total += prod
    return total % q
