"""Failure handling without a GPU fault: a bounded device wait runs out, the
call returns FM_ERR_TIMEOUT with a message, and the context stays usable."""
import numpy as np
import pytest
import scipy.sparse as sp

from feelmri_b200 import _lib as L, ops, workloads as W
from feelmri_b200.MRI import Signal

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_survives(cuda):
    ctx = ops.ctx_for(cuda)
    status = L.lib().fm_selftest_wait(ctx, 1_000_000)  # 1 ms
    assert status == L.FM_ERR_TIMEOUT
    assert "ran out" in L.last_error()
    # the context and the device still work: a normal call succeeds
    mesh = W.cylinder(1500)
    N = mesh.n_nodes
    M = sp.lil_matrix((N, N))
    M.setdiag(np.full(N, 1e-7))
    traj = W.cartesian(res=(4, 8, 4))
    _, T2 = W.tissue(N, 0)
    Mxy = np.ones((N, 1), np.complex64)
    K = Signal(0, M, traj.points, traj.t, mesh.nodes.astype(np.float32), W.off_resonance(N), T2, Mxy, None,
               precision="bf16x3")
    assert np.isfinite(K).all() and np.abs(K).max() > 0


def test_selftest_rejects_bad_limits(cuda):
    ctx = ops.ctx_for(cuda)
    assert L.lib().fm_selftest_wait(ctx, 0) == L.FM_ERR_ARG
    assert L.lib().fm_selftest_wait(ctx, 5_000_000_000) == L.FM_ERR_ARG
