"""CPU oracle of the SumCheck prover path -- test infrastructure, never imported by the product.

``oracle.oracle`` restates the reference's algorithm in Python big integers;
``oracle/sumcheck_oracle.c`` is the same in C for sizes Python cannot reach (built by
``oracle/Makefile`` into ``oracle/_build``). Only tests, the smoke check and the CPU-baseline
leg of bench.py use them, and only as the checker.
"""
