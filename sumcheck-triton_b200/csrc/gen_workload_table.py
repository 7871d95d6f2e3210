"""Emits ``workload_table.h``: the 32 kernel workloads as C++ data for the command-line tool.

Run from the repository root (the build runs it when the header is missing or older):

    python sumcheck-triton_b200/csrc/gen_workload_table.py

The source of truth is ``zkduel_b200.workloads`` (KERNEL_WORKLOADS: name, id and kernel table
order of each workload; WORKLOADS: its expression). Every factor is written as its kernel
table index, so the reference's table fill (value of table v at offset i) lands on the same
variable it does in the reference executable.
"""

from __future__ import annotations

import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "workload_table.h"
sys.path.insert(0, str(HERE.parent))

from zkduel_b200.expression import normalize_expression  # noqa: E402
from zkduel_b200.fields import FIELD_SPECS  # noqa: E402
from zkduel_b200.workloads import KERNEL_WORKLOADS  # noqa: E402


def _poly(terms) -> str:
    out = []
    for c, names in terms:
        body = "*".join(names)
        if c == 1:
            out.append(body)
        elif c == -1:
            out.append("-" + body)
        else:
            out.append(f"{c}*{body}")
    return " + ".join(out).replace("+ -", "- ")


def generate() -> str:
    rows, flat_all, coeffs_all, lens_all = [], [], [], []
    for w in KERNEL_WORKLOADS:
        terms = normalize_expression(w.expression)
        pos = {v: i for i, v in enumerate(w.table_order)}
        t0, f0 = len(lens_all), len(flat_all)
        for c, names in terms:
            coeffs_all.append(int(c))
            lens_all.append(len(names))
            flat_all.extend(pos[n] for n in names)
        degree = max(len(n) for _c, n in terms)
        rows.append(f'    {{"{w.name}", "{_poly(terms)}", {w.ident}, {len(w.table_order)}, {degree}, '
                    f'{len(terms)}, {t0}, {f0}}},')
    fields = []
    for bw in sorted(FIELD_SPECS):
        f = FIELD_SPECS[bw]
        limbs = ", ".join(f"0x{(f.modulus >> (32 * i)) & 0xFFFFFFFF:08x}u" for i in range(f.limbs))
        fields.append(f'    {{"{f.name}", {bw}, {f.limbs}, 0x{f.nprime:08x}u, "{f.modulus:#x}", {{{limbs}}}}},')
    lines = [
        "// GENERATED by gen_workload_table.py from zkduel_b200.workloads -- do not edit by hand.",
        "// The 32 kernel workloads: name, polynomial, id, tables, degree, terms, and where their",
        "// terms start in kTermCoeffs / kTermLens and their factors (kernel table indices) in kFlat.",
        "#pragma once",
        "#include <cstdint>",
        "",
        "namespace sc_cli {",
        "",
        "struct WorkloadDef {",
        "  const char* name;",
        "  const char* poly;",
        "  int id, vars, degree, terms;",
        "  int term0, flat0;",
        "};",
        "",
        f"constexpr int kNumWorkloads = {len(rows)};",
        "constexpr WorkloadDef kWorkloads[] = {",
        *rows,
        "};",
        "constexpr int64_t kTermCoeffs[] = {" + ", ".join(map(str, coeffs_all)) + "};",
        "constexpr int32_t kTermLens[] = {" + ", ".join(map(str, lens_all)) + "};",
        "constexpr int32_t kFlat[] = {" + ", ".join(map(str, flat_all)) + "};",
        "",
        "// The four fields (zkduel_b200.fields.FIELD_SPECS): name, bit width, limbs, -p^-1 mod 2^32,",
        "// modulus in hex, little-endian modulus limbs.",
        "struct FieldDef {",
        "  const char* name;",
        "  int bit_width, limbs;",
        "  uint32_t nprime;",
        "  const char* modulus_hex;",
        "  uint32_t modulus[8];",
        "};",
        f"constexpr int kNumFields = {len(fields)};",
        "constexpr FieldDef kFields[] = {",
        *fields,
        "};",
        "",
        "}  // namespace sc_cli",
        "",
    ]
    return "\n".join(lines)


def main() -> int:
    text = generate()
    if len(sys.argv) > 1 and sys.argv[1] == "--check":
        return 0 if OUT.exists() and OUT.read_text() == text else 1
    OUT.write_text(text)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
