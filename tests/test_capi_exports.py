"""The C-ABI libraries load and export every entry point their headers declare (CPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sparsedirectsolver.jl_b200")


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:sdsb200|sdsa)_[a-z_]+)\s*\(", text)))


@pytest.mark.parametrize("header,lib", [("sdsb200.h", "libsdsb200.so"),
                                        ("sdsb200_analysis.h", "libsdsb200_analysis.so")])
def test_exports(header, lib):
    path = os.path.join(PKG, lib)
    if not os.path.exists(path):
        pytest.fail(f"{lib} is not built (run __graft_entry__.build())")
    so = ctypes.CDLL(path)
    names = declared(header)
    assert len(names) >= 5
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    import sys
    sys.path.insert(0, PKG)
    from sdsb200 import capi
    assert set(capi.EXPORTS) == set(declared("sdsb200.h"))


def test_new_entry_points_reject_a_null_plan():
    """The argument checks come before any device work: a NULL plan is SDSB200_INVALID_VALUE."""
    import sys
    sys.path.insert(0, PKG)
    from sdsb200 import capi

    so = capi.bind(ctypes.CDLL(os.path.join(PKG, "libsdsb200.so")))
    assert so.sdsb200_solve_phase(None, capi.PHASE["fwd"], None, 1, None, 1, 1, None, None) == capi.INVALID_VALUE
    assert b"plan is NULL" in so.sdsb200_last_error()
    assert so.sdsb200_schur_matrix(None, 0, None, 1, 0, None) == capi.INVALID_VALUE


def _c_layout(tmp_path):
    """sizeof and offsetof of the header structs, from the C compiler."""
    import shutil
    import subprocess

    if not shutil.which("gcc"):
        pytest.skip("gcc is missing")
    fields = {
        "sdsb200_symbolic": ["n", "nnz", "ns", "index_width", "structure", "perm", "super_ptr", "snparent", "rowptr",
                             "rowval", "front_ptr", "child_ptr", "child_list", "relind_ptr", "relind", "amap",
                             "amap_ptr", "amap_src", "full_rowptr", "full_colval", "full_srcptr", "full_src",
                             "full_nnz", "full_nsrc", "schur"],
        "sdsb200_plan_options": ["nbatch", "precision", "max_nrhs", "tuning"],
        "sdsb200_opts": ["pivot_type", "pivot_epsilon_alg", "pivot_threshold", "pivot_epsilon", "ir_n_steps",
                         "ir_mode", "ir_tol", "solve_mode", "deterministic_mode"],
        "sdsa_options": ["structure", "view", "index_base", "reordering", "user_perm", "pivot_pairs",
                         "pivot_pair_tolerance", "pivot_threshold", "use_superpanels", "amalg_max_width",
                         "amalg_zero_fraction", "amalg_min_width", "user_pairs", "n_user_pairs",
                         "user_schur_indices"],
        "oracle_symbolic": ["n", "ns", "nnz", "perm", "super_ptr", "snparent", "snpost", "rowptr", "rowval",
                            "front_ptr", "child_ptr", "child_list", "relind_ptr", "relind", "amap", "amap_ptr",
                            "amap_src", "schur"],
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sdsb200.h"', '#include "sdsb200_analysis.h"',
             '#include "oracle.h"', "int main(void) {"]
    for st, fs in fields.items():
        lines.append(f'printf("{st} size %zu\\n", sizeof({st}));')
        for f in fs:
            lines.append(f'printf("{st} {f} %zu\\n", offsetof({st}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "oracle"), str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        st, key, val = line.split()
        layout[(st, key)] = int(val)
    return fields, layout


def test_ctypes_mirrors_match_the_headers(tmp_path):
    """Every ctypes mirror of a header struct has the C layout: the same fields in order, offsets, size
    (the oracle's symbolic struct too, which the checker's ctypes binding fills)."""
    import sys
    sys.path.insert(0, PKG)
    from oracle import oracle
    from sdsb200 import analysis, capi

    fields, layout = _c_layout(tmp_path)
    mirrors = {"sdsb200_symbolic": capi.Symbolic, "sdsb200_plan_options": capi.PlanOptions,
               "sdsb200_opts": capi.Opts, "sdsa_options": analysis._Opts, "oracle_symbolic": oracle._Sym}
    for st, cls in mirrors.items():
        names = [f[0] for f in cls._fields_]
        assert names == fields[st], (st, names)
        assert ctypes.sizeof(cls) == layout[(st, "size")], st
        for f in names:
            assert getattr(cls, f).offset == layout[(st, f)], (st, f)


def test_tuning_encoder_matches_the_header_macros(tmp_path):
    """capi.tuning (and autotune.describe) encode the plan tuning as the header's SDSB200_TUNING* macros."""
    import shutil
    import subprocess
    import sys

    if not shutil.which("gcc"):
        pytest.skip("gcc is missing")
    sys.path.insert(0, PKG)
    from sdsb200.autotune import CANDIDATES, describe
    from sdsb200.capi import tuning

    cases = [(96, 64, 1, 3, 0, 0), (128, 0, 0, 0, 1, 4), (0, 32, 0, 15, 0, 14), (224, 128, 1, 1, 1, 15)]
    lines = ['#include <stdio.h>', '#include "sdsb200.h"', "int main(void) {"]
    for fs, wd, ch, st, steps, sub in cases:
        expr = (f"SDSB200_TUNING_STREAMS({fs}, {wd}, {ch}, {st}) | SDSB200_TUNING_SUBTREE({sub})"
                + (" | SDSB200_TUNING_STEPS" if steps else ""))
        lines.append(f'printf("%d\\n", (int)({expr}));')
    lines.append("return 0; }")
    src = tmp_path / "tuning.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "tuning"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    for case, c_value in zip(cases, out):
        assert tuning(*case) == c_value, case
        d = describe(c_value)
        assert (d["fsmall"], d["wide"], d["chains"], d["streams"], d["steps"], d["subtree"]) == case
    assert all(tuning(*c) >= 0 for c in CANDIDATES)
