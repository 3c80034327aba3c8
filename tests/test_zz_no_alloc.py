"""The allocation-free solve entry point, sdsb200_solve_noalloc (GPU).

Some callers may not allocate device memory once their set-up is over: a
framework whose pool allocator has reserved the device's memory for itself, or a
real-time loop that forbids allocation after start-up. sdsb200_solve keeps its
working vectors in the plan and builds a CUDA graph on the first call with new
buffers, and building that graph allocates. sdsb200_solve_noalloc takes its
working vectors from one fixed static device array of the library instead
(SDSB200_NOALLOC_SCRATCH_BYTES, 32 MiB) and launches the same persistent solve
kernel (the dataflow solve) directly.

These tests call it through the C ABI and compare it with sdsb200_solve (no
refinement) on two calls in a row, within the FP64 tolerance of the other parity
tests (the FP32 tolerance for an FP32 factor, whose solve neither entry point
refines here), and check that sizes beyond the array are refused. The file is named so
that pytest collects it last: a run that stops at the first failure has then
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import rel_max_diff, small_kkt
from sdsb200 import matrices as M

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10   # solutions relative to max(1, max|x|), as the other FP64 parity tests
BERR = 1e-12       # scaled backward error of every FP64 solve
FP32_TOL = 1e-5    # the same for an FP32 factor, unrefined
FP32_BERR = 1e-5   # scaled backward error of an unrefined solve with an FP32 factor
SCRATCH_BYTES = 32 << 20


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _factored(A, structure, **params):
    from sdsb200.solver import DirectSolver

    ds = DirectSolver(A, structure, **params)
    ds.execute("analysis")
    assert ds.execute("factorization") == 0
    return ds


def _noalloc(torch, ds, b, solve_mode=0):
    """X for B = b (n x nrhs, host) through sdsb200_solve_noalloc; returns (rc, X or error text)."""
    from sdsb200._native import numeric_lib

    lib = numeric_lib()
    n = ds.n
    bcm = torch.from_numpy(np.ascontiguousarray(np.asarray(b, np.float64).reshape(n, -1).T)).to(ds.device)
    nrhs = bcm.shape[0]
    xcm = torch.full_like(bcm, float("nan"))
    status = torch.full((1,), 7, dtype=torch.int32, device=ds.device)
    stream = torch.cuda.current_stream(ds.device).cuda_stream
    rc = lib.sdsb200_solve_noalloc(ds._plan, C.c_void_p(xcm.data_ptr()), n, C.c_void_p(bcm.data_ptr()), n, nrhs,
                                   solve_mode, C.c_void_p(status.data_ptr()), C.c_void_p(stream))
    if rc != 0:
        return rc, lib.sdsb200_last_error().decode()
    torch.cuda.synchronize()
    assert int(status.item()) == 0, "a dependency wait of the dataflow solve gave up"
    return rc, xcm.T.cpu().numpy()


def _existing(ds, b, solve_mode=0):
    ds.setparam("solve_mode", solve_mode)
    x = ds.execute("solve", None, b).cpu().numpy().reshape(ds.n, -1)
    ds.setparam("solve_mode", 0)
    return x


CASES = {
    # wide separators (the tiled fronts) and many small fronts
    "SPD": (lambda: M.lap3d(20, 20, 20, seed=6), "SPD", dict(reordering_alg="nd", max_nrhs=3), (0,)),
    # the same with an FP32 factor: the float instance of the solve kernel, unrefined
    "SPD_fp32": (lambda: M.lap3d(20, 20, 20, seed=6), "SPD",
                 dict(reordering_alg="nd", max_nrhs=3, factor_precision="fp32"), (0,)),
    # Bunch-Kaufman LDL^T with 2x2 pivots: the local pivot order and the 2x2 diagonal blocks
    "S": (lambda: small_kkt(22, 22, 200, seed=6), "S", dict(max_nrhs=3), (0,)),
    # threshold-pivoting LU, solves with A and with A^T
    "G": (lambda: M.convection_diffusion3d(12, 12, 12, seed=3), "G",
          dict(pivot_threshold=0.1, reordering_alg="nd", max_nrhs=3), (0, 1)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_matches_solve_twice(torch_cuda, case):
    make, structure, params, modes = CASES[case]
    fp32 = params.get("factor_precision") == "fp32"
    tol, berr = (FP32_TOL, FP32_BERR) if fp32 else (FP64_TOL, BERR)
    A = make()
    ds = _factored(A, structure, **params)
    for mode in modes:
        AA = A.T.tocsr() if mode else A
        # two calls in a row with different right-hand sides: the second finds the first's data in the array
        for seed in (11, 12):
            b = M.rhs(A.shape[0], 3, seed=seed)
            rc, x = _noalloc(torch_cuda, ds, b, mode)
            assert rc == 0, x
            ref = _existing(ds, b, mode)
            assert np.all(np.isfinite(x))
            assert rel_max_diff(x, ref) <= tol
            assert M.scaled_backward_error(AA, x, b) <= berr


def test_noalloc_rejects_sizes_beyond_the_array(torch_cuda):
    # 2 * n * nrhs doubles alone exceed 32 MiB; the fronts stay narrow enough for this many right-hand sides
    A = M.lap2d_shifted(150, 150, seed=1)
    nrhs = 100
    assert 8 * 2 * A.shape[0] * nrhs > SCRATCH_BYTES
    ds = _factored(A, "SPD", reordering_alg="nd", max_nrhs=nrhs)
    rc, msg = _noalloc(torch_cuda, ds, M.rhs(A.shape[0], nrhs, seed=2))
    assert rc == 1, msg   # SDSB200_INVALID_VALUE
    assert "static scratch" in msg
    # the plan is untouched: the allocating entry point still solves, and a small plan still fits
    b = M.rhs(A.shape[0], 2, seed=3)
    assert M.scaled_backward_error(A, _existing(ds, b), b) <= BERR
    small = _factored(M.lap3d(12, 12, 12, seed=2), "SPD", max_nrhs=2)
    b = M.rhs(small.n, 2, seed=4)
    rc, x = _noalloc(torch_cuda, small, b)
    assert rc == 0, x
    assert rel_max_diff(x, _existing(small, b)) <= FP64_TOL
