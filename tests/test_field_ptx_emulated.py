"""The inline-PTX field arithmetic (csrc/field_ptx.cuh, generated, and csrc/field_gold.cuh,
the Goldilocks forms whose carries run on the FMA pipe), checked on the CPU.

Every carry chain in those headers is one asm statement of a small PTX subset. This test parses
each statement and runs it in a Python emulation of those instructions -- 32-bit registers,
one carry flag written by the ``.cc`` forms and read by the ``c`` forms, exactly as the PTX ISA
defines them, with a flag written by a subtraction read only by a subtraction and one written by
an addition or multiply-add read only by those -- then compares the result with big-integer arithmetic: the Montgomery
product a b R^-1 mod p, a + b mod p and a - b mod p, on random and edge operands, for the
reference's four fields and random moduli of each limb count.
"""

from __future__ import annotations

import random
import re
from pathlib import Path

import pytest

CSRC = Path(__file__).resolve().parents[1] / "sumcheck-triton_b200" / "csrc"
HEADER = CSRC / "field_ptx.cuh"
GOLD = CSRC / "field_gold.cuh"
M32 = (1 << 32) - 1

FUNC = re.compile(r"template <> __device__ __forceinline__ void (ptx_\w+)<(\d+)>\((.*?)\) \{\n(.*?)\n\}\n", re.S)


def _parse_asm(body):
    m = re.search(r'asm\((.*?)\n\s*: (.*?)\n\s*: (.*?)\);', body, re.S)
    asm = "".join(re.findall(r'"((?:[^"\\]|\\.)*)"', m.group(1)))
    asm = asm.replace("\\n", "\n").replace("\\t", "")
    outs = re.findall(r'"=&r"\(([^)]*)\)', m.group(2))
    ins = re.findall(r'"r"\(([^)]*)\)', m.group(3))
    lines = [ln.strip() for ln in asm.split("\n")]
    lines = [ln.rstrip(";") for ln in lines if ln and ln not in ("{", "}") and not ln.startswith(".reg")]
    return lines, outs, ins


def _parse_gold():
    text = GOLD.read_text()
    out = {}
    for name, body in re.findall(r"__device__ __forceinline__ void (gold_\w+)\((.*?)\n\}\n", text, re.S):
        out[name] = _parse_asm(body)
    return out


def _parse():
    text = HEADER.read_text()
    out = {}
    for name, L, _sig, body in FUNC.findall(text):
        out[(name, int(L))] = _parse_asm(body)
    return out


def _run(prog, env_in):
    """Runs one parsed asm statement; env_in maps C operand expressions (``a[0]``) to values."""
    lines, outs, ins = prog
    regs = {}
    for k, e in enumerate(ins):
        regs[f"%{len(outs) + k}"] = env_in[e] & M32
    cf = 0
    cf_family = None  # which family last wrote the carry flag: "add" (add/mad .cc) or "sub"

    def val(x):
        if x in regs:
            return regs[x]
        if re.fullmatch(r"-?\d+", x):
            return int(x) & M32
        raise KeyError(f"read of unset register {x}")

    for ln in lines:
        op, rest = ln.split(None, 1)
        args = [a.strip() for a in rest.split(",")]
        d = args[0]
        base = op.split(".")
        if op.startswith("setp.ne"):
            regs[d] = int(val(args[1]) != val(args[2]))
            continue
        if op.startswith("selp"):
            regs[d] = val(args[1]) if val(args[3]) else val(args[2])
            continue
        if op.startswith("mov"):
            regs[d] = val(args[1])
            continue
        if op.startswith("and"):
            regs[d] = val(args[1]) & val(args[2])
            continue
        if op.startswith("min.u32"):
            regs[d] = min(val(args[1]), val(args[2]))
            continue
        cc_out = ".cc" in op
        kind = base[0]
        cin = cf if kind in ("madc", "addc", "subc") else 0
        # The flag means a carry after add / mad and a borrow after sub: reading it across
        # families is not portable (compiled code has given wrong results for it), so a
        # statement that does is rejected.
        if kind in ("madc", "addc"):
            assert cf_family == "add", f"{ln}: reads a carry flag written by a subtraction"
        if kind == "subc":
            assert cf_family == "sub", f"{ln}: reads a carry flag written by an addition"
        if kind in ("mul", "mad", "madc"):
            prod = val(args[1]) * val(args[2])
            part = (prod & M32) if base[1] == "lo" else (prod >> 32)
            s = part if kind == "mul" else part + val(args[3]) + cin
            if cc_out:
                cf, cf_family = s >> 32, "add"
            regs[d] = s & M32
        elif kind in ("add", "addc"):
            s = val(args[1]) + val(args[2]) + cin
            if cc_out:
                cf, cf_family = s >> 32, "add"
            regs[d] = s & M32
        elif kind in ("sub", "subc"):
            s = val(args[1]) - val(args[2]) - cin
            if cc_out:
                cf, cf_family = (1 if s < 0 else 0), "sub"
            regs[d] = s & M32
        else:
            raise ValueError(f"unknown instruction {ln}")
    return [regs[f"%{k}"] for k in range(len(outs))]


PROGS = _parse()
GOLD_PROGS = _parse_gold()
FIELDS = {1: [2**32 - 5], 2: [2**64 - 2**32 + 1], 4: [2**127 - 1],
          8: [0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001]}


def _limbs(x, L):
    return [(x >> (32 * k)) & M32 for k in range(L)]


def _val(ws):
    return sum(w << (32 * k) for k, w in enumerate(ws))


def _env(L, p, a, b):
    env = {f"a[{k}]": w for k, w in enumerate(_limbs(a, L))}
    env.update({f"b[{k}]": w for k, w in enumerate(_limbs(b, L))})
    env.update({f"p[{k}]": w for k, w in enumerate(_limbs(p, L))})
    env["np"] = (-pow(p, -1, 1 << 32)) % (1 << 32)
    return env


def _random_prime(rng, bits):
    while True:
        q = rng.randrange(1 << (bits - 1), 1 << bits) | 1
        if all(pow(w, q - 1, q) == 1 for w in (2, 3, 5, 7)):
            return q


def _moduli(L, eo):
    rng = random.Random(L * 17 + eo)
    out = list(FIELDS[L])
    top = 32 * L - 1 if eo else 32 * L - 2  # even/odd form: p < 2^(32L-1); else the guard's bound
    out += [_random_prime(rng, top), _random_prime(rng, top - 5)]
    if eo and L == 8:
        out.append(2**255 - 19)
    return out


def _operands(p, rng, count):
    edge = [0, 1, 2, p - 1, p - 2, p // 2, p // 3]
    for t in range(count):
        yield (edge[t % len(edge)] if t % 3 == 0 else rng.randrange(p)), rng.randrange(p)


def _low_one_moduli(L):
    """Primes below 2^(32L-1) whose two low words are 1 and 2^32 - 1, as BLS12-381 r's are."""
    rng = random.Random(L * 31)
    out = [q for q in FIELDS[L] if q % 2**64 == 2**64 - 2**32 + 1 and q < 1 << (32 * L - 1)]
    while len(out) < 4:
        q = (rng.randrange(1 << (32 * L - 66), 1 << (32 * L - 65)) << 64) + 2**64 - 2**32 + 1
        if all(pow(w, q - 1, q) == 1 for w in (2, 3, 5, 7)):
            out.append(q)
    return out


@pytest.mark.parametrize("L", [1, 2, 4, 8])
@pytest.mark.parametrize("name", ["ptx_mont_mul", "ptx_mont_mul_eo", "ptx_mont_mul_eo1"])
def test_montgomery_product_chains(name, L):
    if (name, L) not in PROGS:
        pytest.skip(f"{name}<{L}> is not generated")
    eo = "_eo" in name
    for p in (_low_one_moduli(L) if name.endswith("_eo1") else _moduli(L, eo)):
        if eo:
            assert p < 1 << (32 * L - 1)
        rinv = pow(1 << (32 * L), -1, p)
        rng = random.Random(p & 0xFFFF)
        for a, b in _operands(p, rng, 150):
            got = _val(_run(PROGS[(name, L)], _env(L, p, a, b)))
            assert got == a * b * rinv % p, (name, L, hex(p), a, b)


@pytest.mark.parametrize("L", [1, 2, 4, 8])
def test_add_and_sub_chains(L):
    for p in _moduli(L, False):
        rng = random.Random(p & 0xFFF)
        for a, b in _operands(p, rng, 100):
            assert _val(_run(PROGS[("ptx_add_mod", L)], _env(L, p, a, b))) == (a + b) % p
            assert _val(_run(PROGS[("ptx_sub_mod", L)], _env(L, p, a, b))) == (a - b) % p


GOLD_P = 2**64 - 2**32 + 1


@pytest.mark.parametrize("name,op", [
    ("gold_add_fma", lambda a, b: (a + b) % GOLD_P),
    ("gold_sub_fma", lambda a, b: (a - b) % GOLD_P),
    ("gold_mul_fma", lambda a, b: a * b * pow(2**64, -1, GOLD_P) % GOLD_P),
])
def test_goldilocks_fma_pipe_forms(name, op):
    assert name in GOLD_PROGS, sorted(GOLD_PROGS)
    prog = GOLD_PROGS[name]
    x, y = ("x", "y") if name == "gold_mul_fma" else ("a", "b")
    rng = random.Random(len(name))
    edge = [0, 1, 2, GOLD_P - 1, GOLD_P - 2, 2**32, 2**32 - 1, 2**32 + 1, 2**63, GOLD_P // 2]
    for t in range(4000):
        a = edge[t % len(edge)] if t % 3 == 0 else rng.randrange(GOLD_P)
        b = edge[(t // 3) % len(edge)] if t % 5 == 0 else rng.randrange(GOLD_P)
        env = {f"{x}[0]": a & M32, f"{x}[1]": a >> 32, f"{y}[0]": b & M32, f"{y}[1]": b >> 32,
               "k.one": 1, "k.zero": 0, "k.eps": M32}
        assert _val(_run(prog, env)) == op(a, b), (name, a, b)


RINV64 = pow(2**64, -1, GOLD_P)
# the lazy forms: (name, operand names, second operand canonical?, residue of the result)
LAZY = [
    ("gold_add_lazy_c", ("a", "b"), True, lambda a, b: (a + b) % GOLD_P),
    ("gold_add_lazy_c_alu", ("a", "b"), True, lambda a, b: (a + b) % GOLD_P),
    ("gold_add_lazy", ("a", "b"), False, lambda a, b: (a + b) % GOLD_P),
    ("gold_sub_lazy", ("a", "b"), False, lambda a, b: (a - b) % GOLD_P),
    ("gold_mul_any", ("x", "y"), False, lambda a, b: a * b * RINV64 % GOLD_P),
    ("gold_mul_fma", ("x", "y"), False, lambda a, b: a * b * RINV64 % GOLD_P),
]


@pytest.mark.parametrize("name,names,b_canonical,op", LAZY)
def test_goldilocks_lazy_forms(name, names, b_canonical, op):
    """Operands anywhere in [0, 2^64) -- the non-canonical band [p, 2^64) included -- give a
    representative of the right residue (gold_mul_fma too: the lazy kernels use it on any
    operands); gold_mul_any on operands below p equals gold_mul_fma."""
    assert name in GOLD_PROGS, sorted(GOLD_PROGS)
    prog = GOLD_PROGS[name]
    x, y = names
    rng = random.Random(len(name) * 7)
    top = 2**64
    edge = [0, 1, 2, GOLD_P - 1, GOLD_P, GOLD_P + 1, top - 1, top - 2, top - 2**32, 2**32 - 1, 2**32,
            2**63, GOLD_P - 2**32]
    for t in range(6000):
        a = edge[t % len(edge)] if t % 3 == 0 else rng.randrange(top if t % 2 else GOLD_P)
        bmax = GOLD_P if b_canonical else top
        b = edge[(t // 3) % len(edge)] if t % 5 == 0 else rng.randrange(bmax if t % 4 else GOLD_P)
        if b_canonical:
            b %= GOLD_P
        env = {f"{x}[0]": a & M32, f"{x}[1]": a >> 32, f"{y}[0]": b & M32, f"{y}[1]": b >> 32,
               "k.one": 1, "k.zero": 0, "k.eps": M32}
        got = _val(_run(prog, env))
        assert got % GOLD_P == op(a, b), (name, a, b)
        if name == "gold_mul_any" and a < GOLD_P and b < GOLD_P:
            assert got == _val(_run(GOLD_PROGS["gold_mul_fma"], env)) < GOLD_P


def test_goldilocks_canon():
    prog = GOLD_PROGS["gold_canon"]
    rng = random.Random(5)
    vals = [0, 1, GOLD_P - 1, GOLD_P, GOLD_P + 1, 2**64 - 1, 2**64 - 2**32, 2**64 - 2**32 + 2]
    vals += [rng.randrange(2**64) for _ in range(3000)]
    for a in vals:
        env = {"a[0]": a & M32, "a[1]": a >> 32, "k.one": 1, "k.zero": 0, "k.eps": M32}
        assert _val(_run(prog, env)) == a % GOLD_P, a

