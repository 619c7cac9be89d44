"""Sequence driver (BlochSolver) against the reference's block loop restated
on the oracle: per-block timeshift, state carried between blocks, Mxy
spoiled (0 * Mxy) after non-empty blocks, stored columns returned, and
solve(start=-2) continuing from the carried state (Bloch.py:298-380)."""
import numpy as np
import pytest

import oracle
from oracle import fp64
from feelmri_b200 import workloads as W
from feelmri_b200.Bloch import BlochSolver
from feelmri_b200.BlochSimulator import bloch_call_times

pytestmark = pytest.mark.gpu


def _reference_loop(blocks, nodes, T1, T2, dB, pod, Mxy0, Mz0):
    """BlochSolver.solve restated with the oracle (Bloch.py:332-368)."""
    N = nodes.shape[0]
    m, z = Mxy0.astype(np.complex64).copy(), Mz0.astype(np.float32).copy()
    out_m, out_z = [], []
    for b in blocks:
        if pod is not None:
            pod.update_timeshift(b.times[0])
        dt = np.diff(b.times, prepend=0).astype(np.float32)
        disp = None if pod is None else np.stack([pod(t) for t in bloch_call_times(dt)])
        fm, fz = oracle.bloch_f32(nodes, T1, T2, dB, 1.0, np.float32(W.GAMMA), b.rf, b.G, dt, m, z, disp=disp,
                                  history=False)
        if b.store_magnetization:
            out_m.append(fm.copy())
            out_z.append(fz.copy())
        m = fm if b.empty else (0 * fm).astype(np.complex64)
        z = fz
    return np.stack(out_m, 1), np.stack(out_z, 1), m, z


def _blocks():
    blocks = []
    t = 0.0
    for i in range(4):
        b = W.hard_pulse_block(t, 20.0, 4.0, grad=((2.0, -1.0, 0.5), 0.5, 1.0), store=(i % 2 == 1))
        blocks.append(b)
        t += 4.0
        gap = W.hard_pulse_block(t, 0.0, 2.0)
        gap.empty = True
        gap.store_magnetization = (i == 3)
        blocks.append(gap)
        t += 2.0
    return blocks


@pytest.mark.parametrize("with_motion", [False, True])
def test_solver_matches_reference_block_loop(cuda, with_motion):
    mesh = W.cylinder(2500)
    N = mesh.n_nodes
    T1, T2 = W.tissue(N)
    dB = np.zeros(N, np.float32)
    nodes = mesh.nodes.astype(np.float32)
    pod = W.sinusoidal_pod(N, n_modes=3, amp=1e-3, period=12.0, n_frames=7) if with_motion else None
    blocks = _blocks()
    solver = BlochSolver(blocks, nodes, M0=1.0, T1=T1, T2=T2, delta_B=dB, gamma=W.GAMMA, pod_trajectory=pod)
    m, z = solver.solve()
    ref_pod = W.sinusoidal_pod(N, n_modes=3, amp=1e-3, period=12.0, n_frames=7) if with_motion else None
    rm, rz, cm, cz = _reference_loop(blocks, nodes, T1, T2, dB, ref_pod, np.zeros(N), np.ones(N))
    assert m.shape == rm.shape == (N, 3)
    # FP32 rounding differences compound over the 8 chained blocks
    assert fp64.rel_l2(m, rm) < 3e-6
    assert fp64.rel_l2(z, rz) < 3e-6
    np.testing.assert_allclose(solver.initial_Mxy[:, 0], cm, atol=3e-5)
    np.testing.assert_allclose(solver.initial_Mz[:, 0], cz, atol=3e-5)
    # continuing with the last two blocks starts from the carried state
    gm0, gz0 = solver.initial_Mxy[:, 0].copy(), solver.initial_Mz[:, 0].copy()
    m2, z2 = solver.solve(start=-2)
    rm2, rz2, _, _ = _reference_loop(blocks[-2:], nodes, T1, T2, dB, ref_pod, gm0, gz0)
    assert fp64.rel_l2(m2, rm2) < 3e-6
    assert fp64.rel_l2(z2, rz2) < 3e-6
