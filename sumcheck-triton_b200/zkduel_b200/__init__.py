"""B200-native SumCheck prover with the reference's (zkDuel's) surface.

``sumcheck`` / ``available_backends`` / ``get_workload`` / ``WORKLOADS`` keep the names and
meaning of the reference package (``src/zkduel/__init__.py``); ``prove`` is the seeded call
that generates its tables on the device. All proving runs in ``libsumcheck_b200.so``.
"""

from .api import (
    BACKEND,
    CompiledExpression,
    Proof,
    available_backends,
    generate_tables,
    get_context,
    get_device_field,
    prove,
    prove_device,
    sumcheck,
    upload_tables,
)
from .expression import encode_expression, expression_degree, expression_vars, normalize_expression
from .fields import FIELD_SPECS, FieldSpec, UnsafeModulusError, check_montgomery_modulus, get_field
from .transcript import Transcript
from .workloads import KERNEL_WORKLOADS, WORKLOADS, get_kernel_workload, get_workload

__all__ = [
    "BACKEND",
    "CompiledExpression",
    "FIELD_SPECS",
    "FieldSpec",
    "KERNEL_WORKLOADS",
    "Proof",
    "Transcript",
    "UnsafeModulusError",
    "WORKLOADS",
    "available_backends",
    "check_montgomery_modulus",
    "encode_expression",
    "expression_degree",
    "expression_vars",
    "generate_tables",
    "get_context",
    "get_device_field",
    "get_field",
    "get_kernel_workload",
    "get_workload",
    "normalize_expression",
    "prove",
    "prove_device",
    "sumcheck",
    "upload_tables",
]
