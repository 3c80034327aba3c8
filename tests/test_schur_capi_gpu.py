"""Schur complement mode and the solve sub-phases through the C ABI alone.

tests/native/schur_capi_check.cpp drives libsdsb200_analysis.so and libsdsb200.so the way a non-Python
caller would (the reference's Julia extension binds the same entry points): the Schur analysis, the
factorization, sdsb200_schur_matrix, the three Schur phases as sdsb200_solve_phase sequences around a
host solve of the condensed system, and the five sub-phases of a plain plan against sdsb200_solve.
This file writes its cases with dense expectations (numpy), builds it with g++ and runs it on the GPU:
  - "SPD": 2-D Laplacian 10 x 10 with a diagonal shift;
  - "S": the same shifted by -2.5 (indefinite, nonzero diagonal: no perturbed pivot changes S);
  - "G": 3-D convection-diffusion 5^3, for A and for A^T;
with 12 random Schur indices each. Tolerances: S 1e-11, the condensed right-hand side 1e-12, x 1e-10
(all relative to the largest entry); the sub-phases bit for bit against the per-level solve.
"""
import os
import shutil
import struct
import subprocess
import sys

import numpy as np
import pytest
import scipy.sparse as sp

from sdsb200 import matrices as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sparsedirectsolver.jl_b200")
SRC = os.path.join(ROOT, "tests", "native", "schur_capi_check.cpp")
CUDA = "/usr/local/cuda"


def _flags(n, k, seed):
    fl = np.zeros(n, np.int8)
    fl[np.random.default_rng(seed).choice(n, k, replace=False)] = 1
    return fl


def write_cases(path):
    cases = [("SPD", M.lap2d_shifted(10, 10), 0),
             ("S", (M.lap2d_shifted(10, 10) - 2.5 * sp.eye(100)).tocsr(), 0),
             ("G", M.convection_diffusion3d(5, 5, 5, seed=2), 0),
             ("G", M.convection_diffusion3d(5, 5, 5, seed=2), 1)]
    code = {"G": 0, "S": 1, "SPD": 3}
    with open(path, "wb") as fh:
        fh.write(struct.pack("q", len(cases)))
        for st, A, tr in cases:
            A = A.tocsr()
            A.sort_indices()
            n, k = A.shape[0], 12
            fl = _flags(n, k, 7)
            AA = (A.T.tocsr() if tr else A).toarray()
            idx, rest = np.flatnonzero(fl), np.flatnonzero(fl == 0)
            solve11 = lambda r: np.linalg.solve(AA[np.ix_(rest, rest)], r)  # noqa: E731
            Sd = AA[np.ix_(idx, idx)] - AA[np.ix_(idx, rest)] @ solve11(AA[np.ix_(rest, idx)])
            b = np.random.default_rng(11).uniform(-1, 1, n)
            bs = b[idx] - AA[np.ix_(idx, rest)] @ solve11(b[rest])
            x = np.linalg.solve(AA, b)
            fh.write(struct.pack("qqqqqd", n, A.nnz, k, code[st], tr, 0.1 if st == "G" else 0.01))
            for arr, dt in ((A.indptr, np.int64), (A.indices, np.int64), (A.data, np.float64), (fl, np.int8),
                            (Sd.reshape(-1, order="F"), np.float64), (b, np.float64), (bs, np.float64),
                            (x, np.float64)):
                fh.write(np.ascontiguousarray(arr, dtype=dt).tobytes())


def build_check(outdir):
    """Compile the check program against the in-tree libraries (g++; the CUDA runtime's headers only)."""
    exe = os.path.join(outdir, "schur_capi_check")
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           SRC, "-o", exe, "-L", PKG, "-lsdsb200", "-lsdsb200_analysis", "-L", os.path.join(CUDA, "lib64"),
           "-lcudart", f"-Wl,-rpath,{PKG}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def _have_toolchain():
    return shutil.which("g++") and os.path.isdir(os.path.join(CUDA, "include")) and \
        os.path.exists(os.path.join(PKG, "libsdsb200.so")) and os.path.exists(os.path.join(PKG, "libsdsb200_analysis.so"))


def test_schur_capi_check_builds(tmp_path):
    """CPU: the check program compiles and links against the exported C ABI, and its cases are written."""
    if not _have_toolchain():
        pytest.skip("g++, the CUDA headers or the built libraries are missing")
    exe = build_check(str(tmp_path))
    assert os.access(exe, os.X_OK)
    write_cases(str(tmp_path / "cases.bin"))
    assert (tmp_path / "cases.bin").stat().st_size > 0


@pytest.mark.gpu
def test_schur_capi_on_gpu(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    exe = build_check(str(tmp_path))
    cases = str(tmp_path / "cases.bin")
    write_cases(cases)
    r = subprocess.run([exe, cases], capture_output=True, text=True, timeout=120)
    sys.stdout.write(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
