"""Host logic of batches (CPU): block-diagonal assembly, stacking and per-system errors of uneven
batches, and the active-member selection of uniform batches."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from sdsb200 import matrices as M
from sdsb200.batch import UnevenBatch


def test_block_diagonal_and_per_system_errors():
    systems = M.uneven_batch(6, 4, 9, 0.1, 3)
    ub = UnevenBatch(systems, "SPD", device="cpu")
    assert ub.A.shape[0] == sum(A.shape[0] for A in systems)
    for i, A in enumerate(systems):
        o = ub.offsets
        blk = ub.A[o[i]:o[i + 1], o[i]:o[i + 1]]
        assert (abs(blk - A)).max() == 0
    b = ub.stack([np.ones(A.shape[0]) * (i + 1) for i, A in enumerate(systems)])
    x = spla.spsolve(ub.A.tocsc(), b)
    errs = ub.backward_errors(x, b)
    assert errs.shape == (6,) and errs.max() < 1e-14
    # a wrong block shows up in that system only
    x2 = x.copy()
    x2[ub.offsets[2]] += 1.0
    errs2 = ub.backward_errors(x2, b)
    assert errs2[2] > 1e-3 and np.delete(errs2, 2).max() < 1e-14
    parts = ub.split(x)
    assert len(parts) == 6 and all(p.shape[0] == A.shape[0] for p, A in zip(parts, systems))


def test_active_members_restates_the_reference():
    """active_members (src/numeric/batch.jl:115-129): ubatch_index and ubatch_mask together."""
    from sdsb200.solver import InvalidValueError, active_members

    assert active_members(4, -1, None) == [0, 1, 2, 3]
    assert active_members(4, 2, None) == [2]
    assert active_members(4, -1, [1, 0, 1, 1]) == [0, 2, 3]
    assert active_members(4, 2, [1, 0, 1, 1]) == [2]
    assert active_members(4, 1, [1, 0, 1, 1]) == []
    with pytest.raises(InvalidValueError):
        active_members(4, 4, None)
    with pytest.raises(InvalidValueError):
        active_members(4, -2, None)
    with pytest.raises(InvalidValueError):
        active_members(4, -1, [1, 0, 1])
