"""ABI drift check of include/gpuqo_b200.h against the reference's own headers.

The library is a drop-in for the reference's gpuqo object set: a backend
compiled against src/include/optimizer/gpuqo_common.h and
gpuqo_planner_info.h passes its structures to this library, so every struct
must have the same size and member offsets, and both enums the same values.

Three C programs are compiled with gcc:
  * one over the reference's headers and one over this repository's header,
    each printing sizeof / offsetof of every boundary struct member and the
    value of every enum constant; the two listings must be identical;
  * one that includes the reference's headers first and this header after
    them: the header then skips its own type declarations and declares the
    entry point and the GUC variables over the reference's types, so a
    mismatching GUC type or prototype is a compile error.

Needs the reference sources (the oracle Makefile's REF); skipped without them.
"""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ref_include():
    r = subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "print-ref"],
                       capture_output=True, text=True)
    ref = r.stdout.strip()
    inc = os.path.join(ref, "src", "include")
    if r.returncode != 0 or not os.path.isfile(os.path.join(inc, "optimizer", "gpuqo_planner_info.h")):
        pytest.skip("reference sources not present")
    return inc


STRUCTS = {
    "PathCost": ["startup", "total"],
    "GpuqoIndexInfo": ["available", "unique", "rows", "cost"],
    "VarStats": ["stadistinct", "stanullfrac", "mcvfreq"],
    "VarInfo": ["stats", "index"],
    "EqClassInfo": ["eclass", "relids", "sels", "vars", "fk", "next"],
    "BaseRelationC": ["id", "rows", "tuples", "cost", "width"],
    "GpuqoPlannerInfoC": ["n_rels", "base_rels", "edge_table", "eq_classes", "n_eq_classes",
                          "n_eq_class_sels", "n_eq_class_fks", "n_eq_class_vars"],
    "QueryTreeC": ["id", "rows", "cost", "width", "left", "right"],
    "Bitmapset": ["nwords", "words"],
}
ENUMS = ["GPUQO_DPSIZE", "GPUQO_DPSUB", "GPUQO_CPU_DPSIZE", "GPUQO_CPU_DPSUB", "GPUQO_CPU_DPSUB_PARALLEL",
         "GPUQO_CPU_DPSUB_BICC", "GPUQO_CPU_DPSUB_BICC_PARALLEL", "GPUQO_CPU_DPCCP", "GPUQO_DPE_DPSIZE",
         "GPUQO_DPE_DPSUB", "GPUQO_DPE_DPCCP", "GPUQO_CPU_GOO", "GPUQO_CPU_IKKBZ", "GPUQO_CPU_LINEARIZED_DP",
         "GPUQO_CPU_DPLIN", "GPUQO_IDP1", "GPUQO_IDP2", "GPUQO_UNION"]

# what the reference's headers take from Postgres's c.h / pg_config.h
PG_PRELUDE = """
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
typedef uint64_t uint64; typedef int64_t int64; typedef uint32_t uint32; typedef int32_t int32;
#define FLEXIBLE_ARRAY_MEMBER
#define SIZEOF_VOID_P 8
"""
REF_INCLUDES = '#include "nodes/bitmapset.h"\n#include "optimizer/gpuqo_common.h"\n' \
               '#include "optimizer/gpuqo_planner_info.h"\n'


def _listing_source(includes):
    lines = ["#include <stdio.h>", includes, "int main(void) {"]
    for s, fields in STRUCTS.items():
        lines.append(f'printf("sizeof {s} %zu\\n", sizeof({s}));')
        for f in fields:
            lines.append(f'printf("offsetof {s}.{f} %zu\\n", offsetof({s}, {f}));')
    for e in ENUMS:
        lines.append(f'printf("enum {e} %d\\n", (int){e});')
    lines.append("return 0; }")
    return "\n".join(lines)


def _compile_run(tmp_path, name, src, inc_dirs, run=True):
    c = tmp_path / f"{name}.c"
    exe = tmp_path / name
    c.write_text(src)
    out = ["-o", str(exe)] if run else ["-c", "-o", str(exe) + ".o"]
    cmd = ["gcc", "-std=gnu11", "-Wall", "-Werror"] + out + [str(c)] + [f"-I{d}" for d in inc_dirs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    if not run:
        return None
    return subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout


def test_struct_layouts_and_enums_match_reference(tmp_path):
    ref_inc = _ref_include()
    ref = _compile_run(tmp_path, "ref_abi", _listing_source(PG_PRELUDE + REF_INCLUDES), [ref_inc])
    ours = _compile_run(tmp_path, "b200_abi", _listing_source('#include "gpuqo_b200.h"\n'),
                        [os.path.join(REPO, "include")])
    assert ref.splitlines() == ours.splitlines()
    assert len(ref.splitlines()) == len(ENUMS) + sum(1 + len(f) for f in STRUCTS.values())


def test_entry_point_and_gucs_declare_over_reference_types(tmp_path):
    ref_inc = _ref_include()
    src = (PG_PRELUDE + REF_INCLUDES + '#include "gpuqo_b200.h"\n'
           "QueryTreeC *(*volatile entry)(int, GpuqoPlannerInfoC *) = gpuqo_run;\n"
           "int main(void) { return entry == 0; }\n")
    _compile_run(tmp_path, "ref_then_b200", src, [ref_inc, os.path.join(REPO, "include")], run=False)
