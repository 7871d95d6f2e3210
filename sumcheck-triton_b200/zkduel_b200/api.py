"""Public API of the B200 prover.

``sumcheck`` keeps the reference's call (``src/zkduel/api.py:26-64``: host tables keyed by
variable name, modulus, expression, explicit challenges, number of rounds) and returns the
same ``(claim0, round_evals)``; ``prove`` is the north-star call
``(expression, field width, num_vars, seed) -> round polynomials, challenges, final
claims, checksum`` with the tables generated on the device. Both run entirely through
``libsumcheck_b200.so``; there is no CPU backend.
"""

from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass, field as dc_field
from typing import Iterable, Mapping, Sequence

import numpy as np

from . import _lib
from .expression import EncodedExpression, Expression, encode_expression, expression_vars  # noqa: F401
from .fields import FieldSpec, field_for_modulus, from_limbs, get_field

BACKEND = "b200"

_local = threading.local()
_fields: dict[tuple[int, int, int], "DeviceField"] = {}
_fields_lock = threading.Lock()


def _torch():
    import torch

    return torch


def available_backends() -> list[str]:
    """Usable backends: ``["b200"]`` when the library loads and a GPU is visible."""
    try:
        _lib.load()
        torch = _torch()
        if torch.cuda.is_available():
            return [BACKEND]
    except (ImportError, OSError):
        pass
    return []


# --------------------------------------------------------------------------------------
# native handles
# --------------------------------------------------------------------------------------


class Context:
    """An ``sc_ctx``: device, stream and the scratch buffers of the proofs run on it."""

    def __init__(self, device: int, stream_handle: int):
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(lib.sc_ctx_create(int(device), ctypes.c_void_p(stream_handle or None), ctypes.byref(h)), "sc_ctx_create")
        self.handle = h
        self.device = int(device)
        self.stream_handle = stream_handle

    def synchronize(self) -> None:
        _lib.check(_lib.load().sc_ctx_synchronize(self.handle), "sc_ctx_synchronize")

    def set_timing(self, enable: bool) -> None:
        _lib.check(_lib.load().sc_ctx_set_timing(self.handle, int(bool(enable))), "sc_ctx_set_timing")

    def launch_times(self) -> list[float]:
        """Durations (ms) of the round-kernel launches since timing was enabled or last read."""
        lib = _lib.load()
        count = ctypes.c_int(0)
        _lib.check(lib.sc_ctx_launch_times(self.handle, None, 0, ctypes.byref(count)), "sc_ctx_launch_times")
        buf = (ctypes.c_float * max(1, count.value))()
        _lib.check(lib.sc_ctx_launch_times(self.handle, buf, count.value, ctypes.byref(count)), "sc_ctx_launch_times")
        return list(buf)[: count.value]

    def close(self) -> None:
        if self.handle:
            _lib.load().sc_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order varies
        try:
            self.close()
        except Exception:
            pass


def get_context(device=None) -> Context:
    """The calling thread's context for ``device`` on torch's current stream."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    idx = dev.index if dev.index is not None else torch.cuda.current_device()
    stream = torch.cuda.current_stream(idx).cuda_stream
    cache = getattr(_local, "contexts", None)
    if cache is None:
        cache = _local.contexts = {}
    key = (idx, stream)
    if key not in cache:
        with torch.cuda.device(idx):
            cache[key] = Context(idx, stream)
    return cache[key]


class DeviceField:
    """An ``sc_field``: one modulus set up on one device."""

    def __init__(self, spec: FieldSpec, device: int):
        lib = _lib.load()
        h = ctypes.c_void_p()
        torch = _torch()
        with torch.cuda.device(device):
            rc = lib.sc_field_init(spec.limbs, _lib.u32_array(_limbs(spec.modulus, spec.limbs)), spec.nprime, ctypes.byref(h))
        _lib.check(rc, "sc_field_init")
        self.handle = h
        self.spec = spec
        self.device = device

    def __del__(self):  # pragma: no cover
        try:
            if self.handle:
                _lib.load().sc_field_destroy(self.handle)
        except Exception:
            pass


def _limbs(x: int, L: int) -> list[int]:
    return [(int(x) >> (32 * i)) & 0xFFFFFFFF for i in range(L)]


def get_device_field(spec: FieldSpec, device: int) -> DeviceField:
    key = (spec.modulus, spec.limbs, int(device))
    with _fields_lock:
        if key not in _fields:
            _fields[key] = DeviceField(spec, int(device))
        return _fields[key]


class CompiledExpression:
    """An ``sc_expr`` built from an expression's flat encoding."""

    def __init__(self, enc: EncodedExpression, q: int | None = None):
        lib = _lib.load()
        limbs = None
        if any(not (-(1 << 63) <= c < (1 << 63)) for c in enc.coeffs):
            if q is None:
                raise ValueError("coefficients beyond int64 need the modulus")
            words = []
            for c in enc.coeffs:
                words.extend(_limbs(int(c) % int(q), 8))
            limbs = _lib.u32_array(words)
        h = ctypes.c_void_p()
        rc = lib.sc_expr_compile(
            enc.num_vars,
            enc.num_terms,
            _lib.i64_array([c if -(1 << 63) <= c < (1 << 63) else 0 for c in enc.coeffs]),
            limbs,
            _lib.i32_array(enc.term_lens),
            _lib.i32_array(enc.term_offsets),
            _lib.i32_array(enc.flat),
            ctypes.byref(h),
        )
        _lib.check(rc, "sc_expr_compile")
        self.handle = h
        self.encoded = enc

    @property
    def degree(self) -> int:
        return self.encoded.degree

    @property
    def num_vars(self) -> int:
        return self.encoded.num_vars

    def __del__(self):  # pragma: no cover
        try:
            if self.handle:
                _lib.load().sc_expr_destroy(self.handle)
        except Exception:
            pass


# --------------------------------------------------------------------------------------
# results
# --------------------------------------------------------------------------------------


@dataclass
class Proof:
    """Outputs of one proof. ``*_mont`` arrays hold Montgomery limbs (as the transcript and
    checksum see them); the properties decode them to canonical integers."""

    field: FieldSpec
    num_rounds: int
    degree: int
    var_names: tuple[str, ...]
    round_polys_mont: np.ndarray  # (n, d + 1, L) uint32
    challenges_mont: np.ndarray  # (n, L)
    finals_mont: np.ndarray  # (1 + K, L)
    claim0_mont: np.ndarray  # (L,)
    checksum: int
    extras: dict = dc_field(default_factory=dict)

    def _dec(self, limbs) -> int:
        return self.field.decode_limbs([int(x) for x in limbs])

    @property
    def round_polys(self) -> list[list[int]]:
        return [[self._dec(v) for v in row] for row in self.round_polys_mont]

    @property
    def challenges(self) -> list[int]:
        return [self._dec(v) for v in self.challenges_mont]

    @property
    def claim0(self) -> int:
        return self._dec(self.claim0_mont)

    @property
    def final_claim(self) -> int:
        return self._dec(self.finals_mont[0])

    @property
    def final_values(self) -> list[int]:
        return [self._dec(v) for v in self.finals_mont[1:]]


# --------------------------------------------------------------------------------------
# tables
# --------------------------------------------------------------------------------------


def empty_tables(spec: FieldSpec, num_tables: int, num_rounds: int, device=None):
    """Uninitialised limb-planar tables: int32 tensor (K, L, 2^n) on the device."""
    torch = _torch()
    dev = torch.device("cuda") if device is None else torch.device(device)
    return torch.empty((num_tables, spec.limbs, 1 << num_rounds), dtype=torch.int32, device=dev)


def generate_tables(spec: FieldSpec, num_tables: int, num_rounds: int, kinds: Sequence[int], seed: int,
                    device=None, out=None):
    """Seeded tables generated on the device (Montgomery, limb-planar)."""
    ctx = get_context(device)
    fld = get_device_field(spec, ctx.device)
    t = empty_tables(spec, num_tables, num_rounds, ctx.device) if out is None else out
    rc = _lib.load().sc_tables_generate(ctx.handle, fld.handle, int(num_tables), int(num_rounds),
                                        _lib.i32_array(kinds), ctypes.c_uint64(int(seed) & (2**64 - 1)),
                                        ctypes.c_void_p(t.data_ptr()))
    _lib.check(rc, "sc_tables_generate")
    return t


def host_tables_to_limbs(values: Sequence[Sequence[int]] | np.ndarray, spec: FieldSpec) -> np.ndarray:
    """Canonical host tables (K x N, any ints) -> (K, L, N) uint32 limbs of the values mod p."""
    q, L = spec.modulus, spec.limbs
    if isinstance(values, np.ndarray) and values.dtype.kind in "iu" and L <= 2:
        if values.dtype.kind == "i" and (values < 0).any():
            arr = (values.astype(object) % q).astype(np.uint64)
        else:
            arr = values.astype(np.uint64) % np.uint64(q)
        out = np.empty((arr.shape[0], L, arr.shape[1]), dtype=np.uint32)
        out[:, 0, :] = (arr & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        if L == 2:
            out[:, 1, :] = (arr >> np.uint64(32)).astype(np.uint32)
        return out
    rows = [np.array([int(x) % q for x in row], dtype=object) for row in values]
    K, N = len(rows), len(rows[0]) if rows else 0
    out = np.empty((K, L, N), dtype=np.uint32)
    for k, row in enumerate(rows):
        for l in range(L):
            out[k, l, :] = ((row >> (32 * l)) & 0xFFFFFFFF).astype(np.uint32)
    return out


def upload_tables(limbs: np.ndarray, spec: FieldSpec, device=None):
    """(K, L, N) canonical uint32 limbs -> Montgomery tables on the device."""
    torch = _torch()
    ctx = get_context(device)
    fld = get_device_field(spec, ctx.device)
    t = torch.from_numpy(np.ascontiguousarray(limbs).view(np.int32)).to(torch.device("cuda", ctx.device))
    K, _L, N = limbs.shape
    rc = _lib.load().sc_tables_to_mont(ctx.handle, fld.handle, ctypes.c_void_p(t.data_ptr()), ctypes.c_uint64(N), int(K))
    _lib.check(rc, "sc_tables_to_mont")
    return t


def download_tables(t, spec: FieldSpec) -> np.ndarray:
    """Montgomery device tables -> canonical (K, L, N) uint32 limbs on the host (copy)."""
    ctx = get_context(t.device)
    fld = get_device_field(spec, ctx.device)
    c = t.clone()
    K, _L, N = c.shape
    rc = _lib.load().sc_tables_from_mont(ctx.handle, fld.handle, ctypes.c_void_p(c.data_ptr()), ctypes.c_uint64(N), int(K))
    _lib.check(rc, "sc_tables_from_mont")
    return c.cpu().numpy().view(np.uint32)


# --------------------------------------------------------------------------------------
# proving
# --------------------------------------------------------------------------------------


def prove_device(tables, expr: CompiledExpression | Expression, spec: FieldSpec, num_rounds: int,
                 challenge_mode: str = "sha3", challenges: Sequence[int] | None = None,
                 var_names: Sequence[str] | None = None) -> Proof:
    """Prove over device-resident Montgomery tables (``tables``: int32 (K, L, 2^n) tensor)."""
    if not isinstance(expr, CompiledExpression):
        expr = CompiledExpression(encode_expression(expr), spec.modulus)
    enc = expr.encoded
    K, L, n, d = enc.num_vars, spec.limbs, int(num_rounds), enc.degree
    if tuple(tables.shape) != (K, L, 1 << n):
        raise ValueError(f"tables have shape {tuple(tables.shape)}, expected {(K, L, 1 << n)}")
    if not tables.is_contiguous():
        raise ValueError("tables must be contiguous")
    mode = _lib.CHALLENGE_MODES.get(challenge_mode)
    if mode is None:
        raise ValueError(f"challenge_mode must be one of {sorted(_lib.CHALLENGE_MODES)}, got {challenge_mode!r}")
    ctx = get_context(tables.device)
    fld = get_device_field(spec, ctx.device)
    explicit = None
    if mode == _lib.SC_CHALLENGE_EXPLICIT:
        if challenges is None or len(challenges) < n - 1:
            raise ValueError(f"explicit mode needs at least {n - 1} challenges")
        words = []
        for j in range(n):
            c = int(challenges[j]) if j < len(challenges) else 0
            words.extend(spec.montgomery_limbs(c))
        explicit = _lib.u32_array(words)
    polys = np.zeros((n, d + 1, L), dtype=np.uint32)
    chals = np.zeros((n, L), dtype=np.uint32)
    finals = np.zeros((1 + K, L), dtype=np.uint32)
    claim0 = np.zeros((L,), dtype=np.uint32)
    checksum = ctypes.c_uint64(0)
    p = lambda a: a.ctypes.data_as(_lib.U32P)  # noqa: E731
    rc = _lib.load().sc_prove(ctx.handle, fld.handle, expr.handle, n, ctypes.c_void_p(tables.data_ptr()), mode,
                              explicit, p(polys), p(chals), p(finals), p(claim0), ctypes.byref(checksum))
    _lib.check(rc, "sc_prove")
    return Proof(spec, n, d, tuple(var_names or enc.var_names), polys, chals, finals, claim0, int(checksum.value))


def prove_host(host_tables, expr: CompiledExpression | Expression, spec: FieldSpec, num_rounds: int,
               challenge_mode: str = "sha3", challenges: Sequence[int] | None = None, device=None) -> Proof:
    """Prove from canonical host tables: an int32 (K, L, 2^n) tensor of limbs (pinned memory
    for an asynchronous copy) or a uint32 numpy array. Copies them to the device, converts
    them to Montgomery form there and proves; the results come back to the host."""
    torch = _torch()
    if isinstance(host_tables, np.ndarray):
        host_tables = torch.from_numpy(np.ascontiguousarray(host_tables).view(np.int32))
    ctx = get_context(device)
    fld = get_device_field(spec, ctx.device)
    dev = host_tables.to(torch.device("cuda", ctx.device), non_blocking=True)
    K, _L, N = dev.shape
    rc = _lib.load().sc_tables_to_mont(ctx.handle, fld.handle, ctypes.c_void_p(dev.data_ptr()), ctypes.c_uint64(N), int(K))
    _lib.check(rc, "sc_tables_to_mont")
    return prove_device(dev, expr, spec, num_rounds, challenge_mode, challenges)


def prove_launches(expr: CompiledExpression | Expression, spec: FieldSpec, num_rounds: int,
                   device=None) -> tuple[int, int]:
    """(kernel launches, first tail round) of ``prove_device`` for this proof: one launch per
    round before the tail round, then one for all the rest (``sc_prove_launches``)."""
    if not isinstance(expr, CompiledExpression):
        expr = CompiledExpression(encode_expression(expr), spec.modulus)
    ctx = get_context(device)
    fld = get_device_field(spec, ctx.device)
    launches, tail = ctypes.c_int(0), ctypes.c_int(0)
    _lib.check(_lib.load().sc_prove_launches(ctx.handle, fld.handle, expr.handle, int(num_rounds),
                                             ctypes.byref(launches), ctypes.byref(tail)), "sc_prove_launches")
    return launches.value, tail.value


def calibrate_imad(ctx: Context | None = None) -> float:
    """Measured 32-bit multiply-add rate of the device (IMAD/s), the integer-pipe peak."""
    ctx = ctx or get_context()
    out = ctypes.c_double(0.0)
    _lib.check(_lib.load().sc_calibrate_imad(ctx.handle, ctypes.byref(out)), "sc_calibrate_imad")
    return float(out.value)


def sumcheck(
    eval_tables: Mapping[str, Iterable[int] | np.ndarray],
    *,
    q: int,
    expression: Expression,
    challenges: Sequence[int],
    num_rounds: int,
    bit_width: int = 256,
    backend: str = BACKEND,
) -> tuple[int, np.ndarray]:
    """``(claim0, round_evals)`` as the reference's ``zkduel.sumcheck`` returns them.

    Tables are host-side canonical values keyed by variable name; ``challenges[j]`` folds
    round j. Any of the four widths (32/64/128/256) is accepted, with any modulus the
    Montgomery guard accepts at that width.
    """
    if backend != BACKEND:
        raise ValueError(f"Unknown backend: {backend!r}; expected {BACKEND!r}")
    spec = field_for_modulus(int(q), int(bit_width))
    enc = encode_expression(expression)
    n = int(num_rounds)
    size = 1 << n
    rows = []
    for v in enc.var_names:
        t = eval_tables[v]
        arr = t.detach().cpu().numpy() if hasattr(t, "detach") else t
        arr = np.asarray(arr) if isinstance(arr, np.ndarray) else list(arr)
        if len(arr) != size:
            raise ValueError(f"Table for {v!r} has length {len(arr)}, expected {size}")
        rows.append(arr)
    if all(isinstance(r, np.ndarray) and r.dtype.kind in "iu" for r in rows):
        limbs = host_tables_to_limbs(np.stack(rows), spec)
    else:
        limbs = host_tables_to_limbs(rows, spec)
    dev_tables = upload_tables(limbs, spec)
    proof = prove_device(dev_tables, CompiledExpression(enc, spec.modulus), spec, n, "explicit", list(challenges))
    evals = np.array(proof.round_polys, dtype=object)
    return int(proof.claim0), evals


def prove(
    expression: Expression,
    bit_width: int,
    num_vars: int,
    seed: int,
    *,
    table_kinds: Sequence[str] | None = None,
    challenge_mode: str = "sha3",
    challenges: Sequence[int] | None = None,
    arith_index: Sequence[int] | None = None,
    device=None,
) -> Proof:
    """Prove ``expression`` over ``num_vars`` variables on tables generated from ``seed``.

    ``table_kinds[k]`` is ``"uniform"`` (default), ``"bernoulli"`` or ``"arith"`` (the
    reference's fill of table ``arith_index[k]``, default k).
    """
    spec = get_field(bit_width)
    enc = encode_expression(expression)
    K = enc.num_vars
    kinds = []
    for k in range(K):
        kind = "uniform" if table_kinds is None else table_kinds[k]
        if kind == "uniform":
            kinds.append(_lib.SC_TABLE_UNIFORM)
        elif kind == "bernoulli":
            kinds.append(_lib.SC_TABLE_BERNOULLI)
        elif kind == "arith":
            kinds.append(_lib.SC_TABLE_ARITH + (k if arith_index is None else int(arith_index[k])))
        else:
            raise ValueError(f"unknown table kind {kind!r}")
    tables = generate_tables(spec, K, int(num_vars), kinds, seed, device)
    return prove_device(tables, CompiledExpression(enc, spec.modulus), spec, int(num_vars), challenge_mode, challenges)
