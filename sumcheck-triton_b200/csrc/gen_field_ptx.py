"""Emits ``field_ptx.cuh``: the inline-PTX carry chains of the field arithmetic.

Run from the repository root (the build runs it when the header is missing or older):

    python sumcheck-triton_b200/csrc/gen_field_ptx.py

Each operation -- the two-chain Montgomery product (L = 1), the even/odd-chain product
(L = 4, 8; for p < 2^(32 L - 1); also in a form for moduli with p_0 = 1, p_1 = 2^32 - 1),
modular add and subtract (L = 1, 2, 4, 8) -- is ONE asm
statement, generated here as straight-line PTX:

* the carry flag is only meaningful inside one statement (the compiler may place its own
  ``.cc`` instructions between statements), so every chain must be inside one;
* every intermediate lives in a PTX register declared inside the statement, and every
  result operand is early-clobber (``=&r``), so no operand can share a register with a
  value the statement still reads -- the compiler may otherwise merge operands that hold
  equal values (e.g. ``m = t0 * nprime`` when nprime is 1).

Montgomery product (CIOS, Koc-Acar-Kaliski 1996, "Analyzing and comparing Montgomery
multiplication algorithms"), per outer iteration i:

    t += a * b[i]                  two chains: low halves into t[0..L], high halves into t[1..L]
    m  = t[0] * nprime mod 2^32
    t  = (t + m * p) / 2^32        two chains; the one-word shift is a renaming of registers

The accumulator between iterations is L+1 words; the a*b[i] chains therefore drop a carry out
of word L, which is exact whenever (2p-1) + (p-1)(2^32-1) < 2^(32(L+1)) -- the bound the host
guard enforces for every accepted modulus. The m*p chains keep the extra word. One
conditional subtraction brings the result below p.
"""

from __future__ import annotations

import sys
from pathlib import Path

OUT = Path(__file__).resolve().parent / "field_ptx.cuh"


class Asm:
    """Builds one asm statement: PTX lines over named operands and local registers."""

    def __init__(self, outs, ins):
        self.outs = outs  # [(name, c_expr)]
        self.ins = ins  # [(name, c_expr)]
        self.lines = []
        self.locals_u32 = []
        self.locals_pred = []

    def ref(self, name):
        for k, (n, _e) in enumerate(self.outs):
            if n == name:
                return f"%{k}"
        for k, (n, _e) in enumerate(self.ins):
            if n == name:
                return f"%{len(self.outs) + k}"
        return name  # a local register

    def op(self, text, *names):
        self.lines.append(text.format(*[self.ref(n) for n in names]))

    def render(self, indent="    "):
        body = ["{"]
        if self.locals_u32:
            body.append(".reg .u32 " + ", ".join(self.locals_u32) + ";")
        if self.locals_pred:
            body.append(".reg .pred " + ", ".join(self.locals_pred) + ";")
        body += self.lines + ["}"]
        text = ("\\n\\t\"\n" + indent + "    \"").join(body)
        outs = ", ".join(f'"=&r"({e})' for _n, e in self.outs)
        ins = ", ".join(f'"r"({e})' for _n, e in self.ins)
        return f'{indent}asm("{text}"\n{indent}    : {outs}\n{indent}    : {ins});\n'


def gen_mont_mul(L: int) -> str:
    head = (
        f"template <> __device__ __forceinline__ void ptx_mont_mul<{L}>(uint32_t (&r)[{L}], "
        f"const uint32_t (&a)[{L}], const uint32_t (&b)[{L}], const uint32_t (&p)[{L}], uint32_t np) {{\n"
    )
    outs = [(f"r{j}", f"r[{j}]") for j in range(L)]
    ins = [(f"a{j}", f"a[{j}]") for j in range(L)] + [(f"b{j}", f"b[{j}]") for j in range(L)]
    ins += [(f"p{j}", f"p[{j}]") for j in range(L)] + [("np", "np")]
    A = Asm(outs, ins)
    if L == 1:
        A.locals_u32 = ["lo", "hi", "m", "c", "d", "bw"]
        A.locals_pred = ["keep"]
        A.op("mul.lo.u32 lo, {}, {};", "a0", "b0")
        A.op("mul.hi.u32 hi, {}, {};", "a0", "b0")
        A.op("mul.lo.u32 m, lo, {};", "np")
        A.op("mad.lo.cc.u32 lo, m, {}, lo;", "p0")
        A.op("madc.hi.cc.u32 hi, m, {}, hi;", "p0")
        A.op("addc.u32 c, 0, 0;")
        A.op("sub.cc.u32 d, hi, {};", "p0")
        A.op("subc.u32 bw, c, 0;")
        A.op("setp.ne.u32 keep, bw, 0;")
        A.op("selp.b32 {}, hi, d, keep;", "r0")
        return head + A.render() + "}\n\n"
    # physical accumulator registers x0..x{L+1}; logical t[k] is phys[k]
    A.locals_u32 = [f"x{k}" for k in range(L + 2)] + ["m"] + [f"d{k}" for k in range(L)] + ["bw"]
    A.locals_pred = ["keep"]
    phys = [f"x{k}" for k in range(L + 2)]
    # iteration 0: t = a * b0
    for j in range(L):
        A.op(f"mul.lo.u32 {phys[j]}, {{}}, {{}};", f"a{j}", "b0")
    A.op(f"mov.u32 {phys[L]}, 0;")
    for j in range(L):
        op = "mad.hi.cc.u32" if j == 0 else ("madc.hi.u32" if j == L - 1 else "madc.hi.cc.u32")
        A.op(f"{op} {phys[j + 1]}, {{}}, {{}}, {phys[j + 1]};", f"a{j}", "b0")
    for i in range(L):
        if i > 0:
            for j in range(L):
                op = "mad.lo.cc.u32" if j == 0 else "madc.lo.cc.u32"
                A.op(f"{op} {phys[j]}, {{}}, {{}}, {phys[j]};", f"a{j}", f"b{i}")
            A.op(f"addc.u32 {phys[L]}, {phys[L]}, 0;")
            for j in range(L):
                op = "mad.hi.cc.u32" if j == 0 else ("madc.hi.u32" if j == L - 1 else "madc.hi.cc.u32")
                A.op(f"{op} {phys[j + 1]}, {{}}, {{}}, {phys[j + 1]};", f"a{j}", f"b{i}")
        A.op(f"mul.lo.u32 m, {phys[0]}, {{}};", "np")
        for j in range(L):
            op = "mad.lo.cc.u32" if j == 0 else "madc.lo.cc.u32"
            A.op(f"{op} {phys[j]}, m, {{}}, {phys[j]};", f"p{j}")
        A.op(f"addc.cc.u32 {phys[L]}, {phys[L]}, 0;")
        A.op(f"addc.u32 {phys[L + 1]}, 0, 0;")
        for j in range(L):
            op = "mad.hi.cc.u32" if j == 0 else "madc.hi.cc.u32"
            A.op(f"{op} {phys[j + 1]}, m, {{}}, {phys[j + 1]};", f"p{j}")
        A.op(f"addc.u32 {phys[L + 1]}, {phys[L + 1]}, 0;")
        phys = phys[1:] + phys[:1]  # t >>= 32 by renaming: the old t[0] (now zero) becomes t[L+1]
    # final conditional subtraction: t[0..L] < 2p
    for j in range(L):
        op = "sub.cc.u32" if j == 0 else "subc.cc.u32"
        A.op(f"{op} d{j}, {phys[j]}, {{}};", f"p{j}")
    A.op(f"subc.u32 bw, {phys[L]}, 0;")
    A.op("setp.ne.u32 keep, bw, 0;")
    for j in range(L):
        A.op(f"selp.b32 {{}}, {phys[j]}, d{j}, keep;", f"r{j}")
    return head + A.render() + "}\n\n"


def gen_mont_mul_eo(L: int, low_one: bool = False) -> str:
    """Montgomery product with separated even/odd accumulators, for p < 2^(32L-1).

    The products a_j b_i of even j land on word pairs (j, j+1) and those of odd j on
    (j, j+1) with j odd: within each parity no two products share a word, so each parity is
    ONE carry chain with one multiply-add per word (no second pass for the high halves, as
    the two-chain CIOS above needs). The accumulator is t = ev + od 2^32: ev holds words
    0..L-1, od words 1..L. Per outer iteration i:

        ev[0] += ev_old[1]; od = ev_old[2..] + a_odd b_i (the carry of the add flows in);
        ev = od_old + a_even b_i; od[L-1] += carry      (the shift by one word is a renaming)
        m = ev[0] nprime; od += p_odd m; ev += p_even m; od[L-1] += carry

    With t < 2p at every iteration start, t + a b_i + m p < 2p (2^32 + 1) < 2^(32(L+1))
    when p < 2^(32L-1), so no chain carries out of its top word except the two whose carry
    is added explicitly. Finally t = od + ev[1..] < 2p and one conditional subtraction.
    Checked bit for bit against big-integer products (tests/test_gpu_parity.py).

    low_one: the form for moduli whose two low words are p_0 = 1 and p_1 = 2^32 - 1 (the
    BLS12-381 scalar field): nprime = -1, so m = -ev[0], and the three multiplies of a row
    that involve p_0, p_1 and nprime become ALU operations. m p_0 = m is an addition; m p_1 =
    m 2^32 - m has low word -m mod 2^32 = ev[0] and high word m - (m != 0), with m != 0
    exactly when ev[0] != 0. Every row then issues 3 fewer multiply instructions (of 17 for
    L = 8), and the multiplies are what bound the product (the FMA-heavy pipe)."""
    name = "ptx_mont_mul_eo1" if low_one else "ptx_mont_mul_eo"
    head = (
        f"template <> __device__ __forceinline__ void {name}<{L}>(uint32_t (&r)[{L}], "
        f"const uint32_t (&a)[{L}], const uint32_t (&b)[{L}], const uint32_t (&p)[{L}], uint32_t np) {{\n"
    )
    outs = [(f"r{j}", f"r[{j}]") for j in range(L)]
    ins = [(f"a{j}", f"a[{j}]") for j in range(L)] + [(f"b{j}", f"b[{j}]") for j in range(L)]
    ins += [(f"p{j}", f"p[{j}]") for j in range(L)] + [("np", "np")]
    A = Asm(outs, ins)
    # PTX registers are virtual: every iteration's ev and od get fresh names (the shift is a
    # renaming) and the register allocator maps them onto physical registers.
    A.locals_pred = ["keep"]
    A.locals_u32 = ["m", "bw"] + [f"d{k}" for k in range(L)] + [f"t{k}" for k in range(L)]
    if low_one:
        A.locals_u32 += ["nz", "h1"]

    def bank(tag):
        names = [f"{tag}{k}" for k in range(L)]
        A.locals_u32.extend(names)
        return names

    ev, od = bank("e0_"), bank("o0_")
    for i in range(L):
        b = f"b{i}"
        if i == 0:
            for j in range(0, L, 2):
                A.op(f"mul.lo.u32 {ev[j]}, {{}}, {{}};", f"a{j}", b)
                A.op(f"mul.hi.u32 {ev[j + 1]}, {{}}, {{}};", f"a{j}", b)
                A.op(f"mul.lo.u32 {od[j]}, {{}}, {{}};", f"a{j + 1}", b)
                A.op(f"mul.hi.u32 {od[j + 1]}, {{}}, {{}};", f"a{j + 1}", b)
        else:
            ne = list(od)  # the new ev is the old od, one word lower
            no = bank(f"o{i}_")
            A.op(f"add.cc.u32 {ne[0]}, {ne[0]}, {ev[1]};")
            src = ev[2:] + ["0", "0"]
            for j in range(1, L, 2):
                last = j == L - 1
                A.op(f"madc.lo.cc.u32 {no[j - 1]}, {{}}, {{}}, {src[j - 1]};", f"a{j}", b)
                hi = "madc.hi.u32" if last else "madc.hi.cc.u32"
                A.op(f"{hi} {no[j]}, {{}}, {{}}, {src[j]};", f"a{j}", b)
            for j in range(0, L, 2):
                lo = "mad.lo.cc.u32" if j == 0 else "madc.lo.cc.u32"
                A.op(f"{lo} {ne[j]}, {{}}, {{}}, {ne[j]};", f"a{j}", b)
                A.op(f"madc.hi.cc.u32 {ne[j + 1]}, {{}}, {{}}, {ne[j + 1]};", f"a{j}", b)
            A.op(f"addc.u32 {no[L - 1]}, {no[L - 1]}, 0;")
            ev, od = ne, no
        if low_one:
            # m = -ev[0]; m p_1 = (ev[0], m - (ev[0] != 0)); m p_0 = (m, 0)
            A.op(f"sub.u32 m, 0, {ev[0]};")
            A.op(f"min.u32 nz, {ev[0]}, 1;")
            A.op("sub.u32 h1, m, nz;")
            A.op(f"add.cc.u32 {od[0]}, {od[0]}, {ev[0]};")
            A.op(f"addc.cc.u32 {od[1]}, {od[1]}, h1;")
        else:
            A.op(f"mul.lo.u32 m, {ev[0]}, {{}};", "np")
        for j in range(3 if low_one else 1, L, 2):
            lo = "mad.lo.cc.u32" if j == 1 else "madc.lo.cc.u32"
            A.op(f"{lo} {od[j - 1]}, m, {{}}, {od[j - 1]};", f"p{j}")
            A.op(f"madc.hi.cc.u32 {od[j]}, m, {{}}, {od[j]};", f"p{j}")
        if low_one:
            A.op(f"add.cc.u32 {ev[0]}, {ev[0]}, m;")
            A.op(f"addc.cc.u32 {ev[1]}, {ev[1]}, 0;")
        for j in range(2 if low_one else 0, L, 2):
            lo = "mad.lo.cc.u32" if j == 0 else "madc.lo.cc.u32"
            A.op(f"{lo} {ev[j]}, m, {{}}, {ev[j]};", f"p{j}")
            A.op(f"madc.hi.cc.u32 {ev[j + 1]}, m, {{}}, {ev[j + 1]};", f"p{j}")
        A.op(f"addc.u32 {od[L - 1]}, {od[L - 1]}, 0;")
    # t = od + ev[1..]: words 0..L-1, < 2p
    t = [f"t{k}" for k in range(L)]
    A.op(f"add.cc.u32 {t[0]}, {od[0]}, {ev[1]};")
    for k in range(1, L - 1):
        A.op(f"addc.cc.u32 {t[k]}, {od[k]}, {ev[k + 1]};")
    A.op(f"addc.u32 {t[L - 1]}, {od[L - 1]}, 0;")
    for j in range(L):
        op = "sub.cc.u32" if j == 0 else "subc.cc.u32"
        A.op(f"{op} d{j}, {t[j]}, {{}};", f"p{j}")
    A.op("subc.u32 bw, 0, 0;")
    A.op("setp.ne.u32 keep, bw, 0;")
    for j in range(L):
        A.op(f"selp.b32 {{}}, {t[j]}, d{j}, keep;", f"r{j}")
    return head + A.render() + "}\n\n"


def gen_add(L: int) -> str:
    """r = a + b mod p for a, b < p: add chain, trial subtraction, select."""
    head = (
        f"template <> __device__ __forceinline__ void ptx_add_mod<{L}>(uint32_t (&r)[{L}], "
        f"const uint32_t (&a)[{L}], const uint32_t (&b)[{L}], const uint32_t (&p)[{L}]) {{\n"
    )
    outs = [(f"r{j}", f"r[{j}]") for j in range(L)]
    ins = [(f"a{j}", f"a[{j}]") for j in range(L)] + [(f"b{j}", f"b[{j}]") for j in range(L)]
    ins += [(f"p{j}", f"p[{j}]") for j in range(L)]
    A = Asm(outs, ins)
    A.locals_u32 = [f"s{j}" for j in range(L)] + [f"d{j}" for j in range(L)] + ["c", "bw"]
    A.locals_pred = ["keep"]
    for j in range(L):
        op = "add.cc.u32" if j == 0 else "addc.cc.u32"
        A.op(f"{op} s{j}, {{}}, {{}};", f"a{j}", f"b{j}")
    A.op("addc.u32 c, 0, 0;")
    for j in range(L):
        op = "sub.cc.u32" if j == 0 else "subc.cc.u32"
        A.op(f"{op} d{j}, s{j}, {{}};", f"p{j}")
    A.op("subc.u32 bw, c, 0;")
    A.op("setp.ne.u32 keep, bw, 0;")
    for j in range(L):
        A.op(f"selp.b32 {{}}, s{j}, d{j}, keep;", f"r{j}")
    return head + A.render() + "}\n\n"


def gen_sub(L: int) -> str:
    """r = a - b mod p for a, b < p: subtract chain, add p back under the borrow mask."""
    head = (
        f"template <> __device__ __forceinline__ void ptx_sub_mod<{L}>(uint32_t (&r)[{L}], "
        f"const uint32_t (&a)[{L}], const uint32_t (&b)[{L}], const uint32_t (&p)[{L}]) {{\n"
    )
    outs = [(f"r{j}", f"r[{j}]") for j in range(L)]
    ins = [(f"a{j}", f"a[{j}]") for j in range(L)] + [(f"b{j}", f"b[{j}]") for j in range(L)]
    ins += [(f"p{j}", f"p[{j}]") for j in range(L)]
    A = Asm(outs, ins)
    A.locals_u32 = [f"d{j}" for j in range(L)] + [f"q{j}" for j in range(L)] + ["mask"]
    for j in range(L):
        op = "sub.cc.u32" if j == 0 else "subc.cc.u32"
        A.op(f"{op} d{j}, {{}}, {{}};", f"a{j}", f"b{j}")
    A.op("subc.u32 mask, 0, 0;")
    for j in range(L):
        A.op(f"and.b32 q{j}, {{}}, mask;", f"p{j}")
    for j in range(L):
        if L == 1:
            op = "add.u32"
        else:
            op = "add.cc.u32" if j == 0 else ("addc.u32" if j == L - 1 else "addc.cc.u32")
        A.op(f"{op} {{}}, d{j}, q{j};", f"r{j}")
    return head + A.render() + "}\n\n"


def generate() -> str:
    parts = [
        "// GENERATED by gen_field_ptx.py -- do not edit by hand.\n",
        "// Inline-PTX carry chains of the field arithmetic for L = 1, 2, 4, 8 limbs; one asm\n",
        "// statement per operation, intermediates in statement-local registers.\n",
        "#pragma once\n#include <cstdint>\n\n",
        "template <int L> __device__ __forceinline__ void ptx_mont_mul(uint32_t (&r)[L], "
        "const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L], uint32_t np);\n",
        "template <int L> __device__ __forceinline__ void ptx_mont_mul_eo(uint32_t (&r)[L], "
        "const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L], uint32_t np);\n",
        "template <int L> __device__ __forceinline__ void ptx_mont_mul_eo1(uint32_t (&r)[L], "
        "const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L], uint32_t np);\n",
        "template <int L> __device__ __forceinline__ void ptx_add_mod(uint32_t (&r)[L], "
        "const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L]);\n",
        "template <int L> __device__ __forceinline__ void ptx_sub_mod(uint32_t (&r)[L], "
        "const uint32_t (&a)[L], const uint32_t (&b)[L], const uint32_t (&p)[L]);\n\n",
    ]
    for L in (1, 2, 4, 8):
        parts.append(f"// ---------------- L = {L} ----------------\n")
        # The two-chain product is the kernels' choice at one limb only; from two limbs up the
        # special reductions, the C++ CIOS or the even/odd form measured faster (field.cuh).
        if L == 1:
            parts.append(gen_mont_mul(L))
        if L >= 4:
            parts.append(gen_mont_mul_eo(L))
            parts.append(gen_mont_mul_eo(L, low_one=True))
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
