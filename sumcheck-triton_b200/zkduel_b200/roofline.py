"""Algorithmic work of a round-kernel launch (the roofline numerators).

For round j of a proof with K tables, degree d, N_j = 2^(n - j) entries per table after the
fold and M = sum over terms of (term length - 1) products per point:

  bytes(j) = K N_0 4L                      j = 0 (read the tables once)
           = K (N_{j-1} + N_j) 4L           j >= 1 (read T_{j-1}, write T_j) = 3 K N_j 4L
  imad(j)  = c_L [ (N_j / 2)(d + 1) M + (j >= 1) K N_j ],  c_L = 2 (2 L^2 + L)

c_L is the multiply-add count of one L-limb CIOS product. Summed over the rounds these are
the whole-proof figures K B (4N - 6) and c_L [(N - 1)(d + 1) M + K (N - 2)] (B = 4L bytes).
Algebraic savings a kernel makes (skipping a point, factoring a table out of every term)
do not lower the numerator; they show up as a higher achieved rate.
"""

from __future__ import annotations


def cios_imad(L: int) -> int:
    return 2 * (2 * L * L + L)


def products_per_point(expression_terms) -> int:
    return sum(len(f) - 1 for _c, f in expression_terms)


def launch_bytes(K: int, L: int, n: int, j: int) -> int:
    nj = 1 << (n - j)
    return K * nj * 4 * L if j == 0 else 3 * K * nj * 4 * L


def launch_imad(K: int, L: int, d: int, M: int, n: int, j: int) -> int:
    nj = 1 << (n - j)
    return cios_imad(L) * ((nj // 2) * (d + 1) * M + (K * nj if j else 0))


def proof_bytes(K: int, L: int, n: int) -> int:
    return sum(launch_bytes(K, L, n, j) for j in range(n))


def proof_imad(K: int, L: int, d: int, M: int, n: int) -> int:
    return sum(launch_imad(K, L, d, M, n, j) for j in range(n))
