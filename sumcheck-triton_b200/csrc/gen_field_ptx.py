"""Emits ``field_ptx.cuh``: the inline-PTX carry chains of the field arithmetic.

Run from the repository root (the build runs it when the header is missing or older):

    python sumcheck-triton_b200/csrc/gen_field_ptx.py

Why a generator: every carry chain (``add.cc``/``addc``, ``mad.lo.cc``/``madc.hi.cc``) must sit
inside ONE ``asm`` statement, because the carry flag is not preserved across statements
(the compiler may schedule its own ``.cc`` instructions in between). A chain is as long as the
limb count, so each limb count L in {1, 2, 4, 8} gets its own unrolled statements. Every
chain emitted here ends in an instruction without ``.cc``, so no carry is live between
statements.

Montgomery product (CIOS, Koc-Acar-Kaliski 1996, "Analyzing and comparing Montgomery
multiplication algorithms"), per outer iteration i:

    t += a * b[i]                  two chains: low halves into t[0..L], high halves into t[1..L]
    m  = t[0] * nprime mod 2^32
    t  = (t + m * p) / 2^32        two chains, then a one-word shift

The accumulator between iterations is L+1 words; the a*b[i] chains therefore drop a carry out
of word L, which is exact whenever (2p-1) + (p-1)(2^32-1) < 2^(32(L+1)) -- the bound the host
guard enforces for every accepted modulus. The m*p chains keep the extra word. One
conditional subtraction brings the result below p.
"""

from __future__ import annotations

import sys
from pathlib import Path

OUT = Path(__file__).resolve().parent / "field_ptx.cuh"


def _asm(lines, outs, ins):
    """One asm statement: lines use {o0..}/{i0..} placeholders for operands."""
    nout = len(outs)
    body = []
    for ln in lines:
        for k in range(len(outs)):
            ln = ln.replace(f"{{o{k}}}", f"%{k}")
        for k in range(len(ins)):
            ln = ln.replace(f"{{i{k}}}", f"%{nout + k}")
        body.append(ln)
    text = "\\n\\t\"\n        \"".join(body)
    o = ", ".join(outs)
    i = ", ".join(ins)
    return f'    asm(\n        "{text}"\n        : {o}\n        : {i});\n'


def gen_mont_mul(L: int) -> str:
    """CIOS with an (L+1)-word accumulator t[0..L] and a transient t[L+1]."""
    s = []
    s.append(
        f"template <> __device__ __forceinline__ void ptx_mont_mul<{L}>(uint32_t (&r)[{L}], "
        f"const uint32_t (&a)[{L}], const uint32_t (&b)[{L}], const uint32_t (&p)[{L}], "
        f"uint32_t np) {{\n"
    )
    if L == 1:
        s.append("    uint32_t hi, c;\n")
        s.append(
            _asm(
                [
                    "{",
                    ".reg .u32 lo, m;",
                    "mul.lo.u32 lo, {i0}, {i1};",
                    "mul.hi.u32 {o0}, {i0}, {i1};",
                    "mul.lo.u32 m, lo, {i3};",
                    "mad.lo.cc.u32 lo, m, {i2}, lo;",
                    "madc.hi.cc.u32 {o0}, m, {i2}, {o0};",
                    "addc.u32 {o1}, 0, 0;",
                    "}",
                ],
                ['"=&r"(hi)', '"=&r"(c)'],
                ['"r"(a[0])', '"r"(b[0])', '"r"(p[0])', '"r"(np)'],
            )
        )
        s.append("    uint32_t d, bw;\n")
        s.append(
            _asm(
                ["sub.cc.u32 {o0}, {i0}, {i2};", "subc.u32 {o1}, {i1}, 0;"],
                ['"=&r"(d)', '"=&r"(bw)'],
                ['"r"(hi)', '"r"(c)', '"r"(p[0])'],
            )
        )
        s.append("    r[0] = bw ? hi : d;\n}\n\n")
        return "".join(s)

    s.append(f"    uint32_t t[{L + 2}];\n")
    # iteration 0: t = a * b[0] (no accumulate)
    lo = [f"mul.lo.u32 {{o{j}}}, {{i{j}}}, {{i{L}}};" for j in range(L)]
    lo.append(f"mov.u32 {{o{L}}}, 0;")
    s.append(
        _asm(
            lo,
            [f'"=&r"(t[{j}])' for j in range(L + 1)],
            [f'"r"(a[{j}])' for j in range(L)] + ['"r"(b[0])'],
        )
    )
    hi = []
    for j in range(L):
        op = "mad.hi.cc.u32" if j == 0 else ("madc.hi.u32" if j == L - 1 else "madc.hi.cc.u32")
        hi.append(f"{op} {{o{j + 1}}}, {{i{j}}}, {{i{L}}}, {{o{j + 1}}};")
    s.append(
        _asm(
            hi,
            [f'"+r"(t[{j}])' for j in range(L + 1)],
            [f'"r"(a[{j}])' for j in range(L)] + ['"r"(b[0])'],
        )
    )
    s.append("#pragma unroll\n")
    s.append(f"    for (int i = 0; i < {L}; ++i) {{\n")
    s.append("      if (i > 0) {\n")
    # t += a * b[i]: low halves
    lo = []
    for j in range(L):
        op = "mad.lo.cc.u32" if j == 0 else "madc.lo.cc.u32"
        lo.append(f"{op} {{o{j}}}, {{i{j}}}, {{i{L}}}, {{o{j}}};")
    lo.append(f"addc.u32 {{o{L}}}, {{o{L}}}, 0;")
    s.append(
        _asm(
            lo,
            [f'"+r"(t[{j}])' for j in range(L + 1)],
            [f'"r"(a[{j}])' for j in range(L)] + ['"r"(b[i])'],
        ).replace("\n    ", "\n      ").replace("    asm", "      asm", 1)
    )
    hi = []
    for j in range(L):
        op = "mad.hi.cc.u32" if j == 0 else ("madc.hi.u32" if j == L - 1 else "madc.hi.cc.u32")
        hi.append(f"{op} {{o{j + 1}}}, {{i{j}}}, {{i{L}}}, {{o{j + 1}}};")
    s.append(
        _asm(
            hi,
            [f'"+r"(t[{j}])' for j in range(L + 1)],
            [f'"r"(a[{j}])' for j in range(L)] + ['"r"(b[i])'],
        ).replace("\n    ", "\n      ").replace("    asm", "      asm", 1)
    )
    s.append("      }\n")
    s.append("      const uint32_t m = t[0] * np;\n")
    # t += m * p: low halves (t[0] becomes 0), carry into t[L], t[L+1]
    lo = []
    for j in range(L):
        op = "mad.lo.cc.u32" if j == 0 else "madc.lo.cc.u32"
        lo.append(f"{op} {{o{j}}}, {{i{L}}}, {{i{j}}}, {{o{j}}};")
    lo.append(f"addc.cc.u32 {{o{L}}}, {{o{L}}}, 0;")
    lo.append(f"addc.u32 {{o{L + 1}}}, 0, 0;")
    s.append(
        _asm(
            lo,
            [f'"+r"(t[{j}])' for j in range(L + 1)] + [f'"=&r"(t[{L + 1}])'],
            [f'"r"(p[{j}])' for j in range(L)] + ['"r"(m)'],
        ).replace("\n    ", "\n      ").replace("    asm", "      asm", 1)
    )
    hi = []
    for j in range(L):
        op = "mad.hi.cc.u32" if j == 0 else "madc.hi.cc.u32"
        hi.append(f"{op} {{o{j + 1}}}, {{i{L}}}, {{i{j}}}, {{o{j + 1}}};")
    hi.append(f"addc.u32 {{o{L + 1}}}, {{o{L + 1}}}, 0;")
    s.append(
        _asm(
            hi,
            [f'"+r"(t[{j}])' for j in range(L + 2)],
            [f'"r"(p[{j}])' for j in range(L)] + ['"r"(m)'],
        ).replace("\n    ", "\n      ").replace("    asm", "      asm", 1)
    )
    s.append("#pragma unroll\n")
    s.append(f"      for (int j = 0; j <= {L}; ++j) t[j] = t[j + 1];\n")
    s.append("    }\n")
    # final conditional subtraction: t[0..L] < 2p
    s.append(f"    uint32_t d[{L}], bw;\n")
    sub = []
    for j in range(L):
        op = "sub.cc.u32" if j == 0 else "subc.cc.u32"
        sub.append(f"{op} {{o{j}}}, {{i{j}}}, {{i{L + 1 + j}}};")
    sub.append(f"subc.u32 {{o{L}}}, {{i{L}}}, 0;")
    s.append(
        _asm(
            sub,
            [f'"=&r"(d[{j}])' for j in range(L)] + ['"=&r"(bw)'],
            [f'"r"(t[{j}])' for j in range(L + 1)] + [f'"r"(p[{j}])' for j in range(L)],
        )
    )
    s.append("#pragma unroll\n")
    s.append(f"    for (int j = 0; j < {L}; ++j) r[j] = bw ? t[j] : d[j];\n")
    s.append("}\n\n")
    return "".join(s)


def gen_add(L: int) -> str:
    """r = a + b mod p for a, b < p: add chain, trial subtraction, select."""
    s = [
        f"template <> __device__ __forceinline__ void ptx_add_mod<{L}>(uint32_t (&r)[{L}], "
        f"const uint32_t (&a)[{L}], const uint32_t (&b)[{L}], const uint32_t (&p)[{L}]) {{\n",
        f"    uint32_t s[{L}], d[{L}], c, bw;\n",
    ]
    lines = []
    for j in range(L):
        op = "add.cc.u32" if j == 0 else "addc.cc.u32"
        lines.append(f"{op} {{o{j}}}, {{i{j}}}, {{i{L + j}}};")
    lines.append(f"addc.u32 {{o{L}}}, 0, 0;")
    s.append(
        _asm(
            lines,
            [f'"=&r"(s[{j}])' for j in range(L)] + ['"=&r"(c)'],
            [f'"r"(a[{j}])' for j in range(L)] + [f'"r"(b[{j}])' for j in range(L)],
        )
    )
    lines = []
    for j in range(L):
        op = "sub.cc.u32" if j == 0 else "subc.cc.u32"
        lines.append(f"{op} {{o{j}}}, {{i{j}}}, {{i{L + 1 + j}}};")
    lines.append(f"subc.u32 {{o{L}}}, {{i{L}}}, 0;")
    s.append(
        _asm(
            lines,
            [f'"=&r"(d[{j}])' for j in range(L)] + ['"=&r"(bw)'],
            [f'"r"(s[{j}])' for j in range(L)] + ['"r"(c)'] + [f'"r"(p[{j}])' for j in range(L)],
        )
    )
    s.append("#pragma unroll\n")
    s.append(f"    for (int j = 0; j < {L}; ++j) r[j] = bw ? s[j] : d[j];\n")
    s.append("}\n\n")
    return "".join(s)


def gen_sub(L: int) -> str:
    """r = a - b mod p for a, b < p: subtract chain, add p back under the borrow mask."""
    s = [
        f"template <> __device__ __forceinline__ void ptx_sub_mod<{L}>(uint32_t (&r)[{L}], "
        f"const uint32_t (&a)[{L}], const uint32_t (&b)[{L}], const uint32_t (&p)[{L}]) {{\n",
        f"    uint32_t d[{L}], mask, q[{L}];\n",
    ]
    lines = []
    for j in range(L):
        op = "sub.cc.u32" if j == 0 else "subc.cc.u32"
        lines.append(f"{op} {{o{j}}}, {{i{j}}}, {{i{L + j}}};")
    lines.append(f"subc.u32 {{o{L}}}, 0, 0;")
    s.append(
        _asm(
            lines,
            [f'"=&r"(d[{j}])' for j in range(L)] + ['"=&r"(mask)'],
            [f'"r"(a[{j}])' for j in range(L)] + [f'"r"(b[{j}])' for j in range(L)],
        )
    )
    s.append("#pragma unroll\n")
    s.append(f"    for (int j = 0; j < {L}; ++j) q[j] = p[j] & mask;\n")
    lines = []
    for j in range(L):
        op = "add.cc.u32" if j == 0 else ("addc.u32" if j == L - 1 else "addc.cc.u32")
        if L == 1:
            op = "add.u32"
        lines.append(f"{op} {{o{j}}}, {{i{j}}}, {{i{L + j}}};")
    s.append(
        _asm(
            lines,
            [f'"=&r"(r[{j}])' for j in range(L)],
            [f'"r"(d[{j}])' for j in range(L)] + [f'"r"(q[{j}])' for j in range(L)],
        )
    )
    s.append("}\n\n")
    return "".join(s)


def generate() -> str:
    parts = [
        "// GENERATED by gen_field_ptx.py -- do not edit by hand.\n",
        "// Inline-PTX carry chains of the field arithmetic for L = 1, 2, 4, 8 limbs.\n",
        "#pragma once\n#include <cstdint>\n\n",
        "template <int L> __device__ __forceinline__ void ptx_mont_mul(uint32_t (&r)[L], "
        "const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L], uint32_t np);\n",
        "template <int L> __device__ __forceinline__ void ptx_add_mod(uint32_t (&r)[L], "
        "const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L]);\n",
        "template <int L> __device__ __forceinline__ void ptx_sub_mod(uint32_t (&r)[L], "
        "const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L]);\n\n",
    ]
    for L in (1, 2, 4, 8):
        parts.append(f"// ---------------- L = {L} ----------------\n")
        parts.append(gen_mont_mul(L))
        parts.append(gen_add(L))
        parts.append(gen_sub(L))
    return "".join(parts)


def main() -> int:
    text = generate()
    if len(sys.argv) > 1 and sys.argv[1] == "--check":
        return 0 if OUT.exists() and OUT.read_text() == text else 1
    OUT.write_text(text)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
