"""Suspending and resuming a proof: transcripts (``sc_transcript_*``, ``sc_prove_resume``).

A :class:`Transcript` is a proof stopped at a round boundary: a flat array of u32 words
(header, then the prover's state after its last round) that can be stored anywhere --
``to_bytes`` / ``from_bytes``, ``save`` / ``load`` -- and continued later from the same
tables, by :func:`prove_rounds` on any GPU or by a server (``ProofServer.submit(...,
resume=t)``), with results bit-identical to the uninterrupted proof. The reference has no
counterpart: its proofs run start to finish inside one call (src/zkduel/api.py:26-64).

    t = start(expr, spec, n)
    t = prove_rounds(tables, expr, spec, 8, t)      # rounds 0..7
    blob = t.to_bytes()                              # ... store, restart, load ...
    t = prove_rounds(tables, expr, spec, n, Transcript.from_bytes(blob))
    proof = result(t, expr, spec)                    # == prove_device(tables, expr, spec, n)
"""

from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Sequence

import numpy as np

from . import _lib
from .api import CompiledExpression, Proof, get_context, get_device_field
from .expression import encode_expression
from .fields import FieldSpec

HEADER_WORDS = 16
MAGIC = 0x31524353  # "SCR1"
MODES = {v: k for k, v in _lib.CHALLENGE_MODES.items()}


def _compiled(expression, spec: FieldSpec) -> CompiledExpression:
    if isinstance(expression, CompiledExpression):
        return expression
    return CompiledExpression(encode_expression(expression), spec.modulus)


class Transcript:
    """A proof's transcript words (uint32, little-endian when serialised). The header is
    checked by the library (``sc_transcript_info``) on construction; no GPU is needed."""

    def __init__(self, words):
        w = np.ascontiguousarray(np.asarray(words, dtype=np.uint32)).copy()
        n, done, mode, tag = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_uint64(0)
        rc = _lib.load().sc_transcript_info(w.ctypes.data_as(_lib.U32P), w.size, ctypes.byref(n), ctypes.byref(done),
                                            ctypes.byref(mode), ctypes.byref(tag))
        _lib.check(rc, "sc_transcript_info")
        self.words = w
        self.num_rounds = n.value
        self.rounds_done = done.value
        self.challenge_mode = MODES[mode.value]
        self.tables_tag = int(tag.value)

    @property
    def complete(self) -> bool:
        return self.rounds_done == self.num_rounds

    def to_bytes(self) -> bytes:
        return self.words.astype("<u4").tobytes()

    @classmethod
    def from_bytes(cls, blob: bytes) -> "Transcript":
        return cls(np.frombuffer(blob, dtype="<u4"))

    def save(self, path) -> None:
        Path(path).write_bytes(self.to_bytes())

    @classmethod
    def load(cls, path) -> "Transcript":
        return cls.from_bytes(Path(path).read_bytes())

    def __repr__(self) -> str:
        return (f"Transcript(rounds {self.rounds_done}/{self.num_rounds}, {self.challenge_mode}, "
                f"{self.words.size} words)")


def tables_tag(kinds: Sequence[int], seed: int) -> int:
    """The tag of ``generate_tables(spec, len(kinds), n, kinds, seed)``'s tables, as the
    server records it (``sc_tables_tag``)."""
    out = ctypes.c_uint64(0)
    k = _lib.i32_array(kinds)
    _lib.check(_lib.load().sc_tables_tag(len(kinds), k, ctypes.c_uint64(int(seed)), ctypes.byref(out)), "sc_tables_tag")
    return int(out.value)


def start(expression, spec: FieldSpec, num_rounds: int, challenge_mode: str = "sha3", tables_tag: int = 0,
          device=None) -> Transcript:
    """A transcript with no rounds done."""
    expr = _compiled(expression, spec)
    fld = get_device_field(spec, get_context(device).device)
    lib = _lib.load()
    words = ctypes.c_uint64(0)
    _lib.check(lib.sc_transcript_words(fld.handle, expr.handle, int(num_rounds), ctypes.byref(words)),
               "sc_transcript_words")
    mode = _lib.CHALLENGE_MODES.get(challenge_mode)
    if mode is None:
        raise ValueError(f"challenge_mode must be one of {sorted(_lib.CHALLENGE_MODES)}, got {challenge_mode!r}")
    w = np.zeros(words.value, dtype=np.uint32)
    rc = lib.sc_transcript_init(fld.handle, expr.handle, int(num_rounds), mode, ctypes.c_uint64(int(tables_tag)),
                                w.ctypes.data_as(_lib.U32P), w.size)
    _lib.check(rc, "sc_transcript_init")
    return Transcript(w)


def prove_rounds(tables, expression, spec: FieldSpec, stop_round: int, transcript: Transcript,
                 challenges: Sequence[int] | None = None) -> Transcript:
    """Rounds [transcript.rounds_done, stop_round) over device tables T_0 (int32 (K, L, 2^n)
    tensor, as for ``prove_device``); returns the longer transcript (the argument is left
    as it was). Explicit mode: ``challenges`` holds every round's challenge."""
    expr = _compiled(expression, spec)
    n = transcript.num_rounds
    K, L = expr.num_vars, spec.limbs
    if tuple(tables.shape) != (K, L, 1 << n) or not tables.is_contiguous():
        raise ValueError(f"tables have shape {tuple(tables.shape)}, expected contiguous {(K, L, 1 << n)}")
    ctx = get_context(tables.device)
    fld = get_device_field(spec, ctx.device)
    explicit = None
    if transcript.challenge_mode == "explicit":
        if challenges is None or len(challenges) < n - 1:
            raise ValueError(f"explicit mode needs at least {n - 1} challenges")
        ws = []
        for j in range(n):
            ws.extend(spec.montgomery_limbs(int(challenges[j]) if j < len(challenges) else 0))
        explicit = _lib.u32_array(ws)
    w = transcript.words.copy()
    rc = _lib.load().sc_prove_resume(ctx.handle, fld.handle, expr.handle, ctypes.c_void_p(tables.data_ptr()), explicit,
                                     int(stop_round), w.ctypes.data_as(_lib.U32P), w.size)
    _lib.check(rc, "sc_prove_resume")
    return Transcript(w)


def result(transcript: Transcript, expression, spec: FieldSpec, var_names: Sequence[str] | None = None) -> Proof:
    """The proof of a complete transcript (``sc_transcript_result``)."""
    expr = _compiled(expression, spec)
    fld = get_device_field(spec, get_context().device)
    n, d, L, K = transcript.num_rounds, expr.degree, spec.limbs, expr.num_vars
    polys = np.zeros((n, d + 1, L), dtype=np.uint32)
    chals = np.zeros((n, L), dtype=np.uint32)
    finals = np.zeros((1 + K, L), dtype=np.uint32)
    claim0 = np.zeros((L,), dtype=np.uint32)
    cs = ctypes.c_uint64(0)
    p = lambda a: a.ctypes.data_as(_lib.U32P)  # noqa: E731
    w = transcript.words
    rc = _lib.load().sc_transcript_result(fld.handle, expr.handle, p(w), w.size, p(polys), p(chals), p(finals),
                                          p(claim0), ctypes.byref(cs))
    _lib.check(rc, "sc_transcript_result")
    return Proof(spec, n, d, tuple(var_names or expr.encoded.var_names), polys, chals, finals, claim0, int(cs.value))
