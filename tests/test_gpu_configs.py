"""Parity of the CUDA paths at the benchmark configurations' sizes.

* plain (config 0): the full ~20k-node cylinder with a 20-pulse spoiled GRE
  (15 degrees, TR 5 ms) and a 64 x 64 Cartesian readout -- the Bloch sweep
  through BlochSolver against the FP32 restatement of the reference's block
  loop, and the FP64 Signal overload against the FP64 restatement (the
  reference's float-rounded pi) at <= 1e-12;
* phase-contrast flow (config 1): the full 200k-node tube with its flow
  motion and 96 x 96 x 32 readout, 4 encoding columns -- the FP32 and
  split-BF16 forms against the float64 direct sum on 1,000 seeded samples
  (<= 1e-5 and <= 1e-4);
* precision (config 2) with fewer nodes: 3-D radial to |k| = 500 1/m, rank-10
  mode motion, 8 coils -- split-BF16 against the float64 direct sum (<= 1e-4).
"""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from oracle import fp64
from feelmri_b200 import workloads as W
from feelmri_b200.MRI import Signal, signal_call_times

pytestmark = pytest.mark.gpu


def _lumped(mesh, dtype=np.float64):
    from feelmri_b200.Assemble import mass_lumped
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    return np.asarray(mass_lumped(mesh.elems, mesh.nodes.astype(dtype), FiniteElement(), QuadratureRule(order=2)))


def test_plain_config_full_size(cuda):
    from feelmri_b200.Bloch import BlochSolver
    mesh = W.cylinder(20_000)
    N = mesh.n_nodes
    assert 19_000 <= N <= 21_000
    T1, T2 = W.tissue(N, 0)
    blocks = W.spoiled_gre(20, 15.0, 5.0)
    nodes32 = mesh.nodes.astype(np.float32)
    m, z = BlochSolver(blocks, nodes32, None, 1.0, T1, T2).solve()
    assert m.shape == (N, 1)
    # the reference's block loop on the FP32 restatement: state carried, Mxy
    # spoiled after every non-empty block (Bloch.py:332-368)
    mm, zz = np.zeros(N, np.complex64), np.ones(N, np.float32)
    from feelmri_b200.Bloch import DEFAULT_GAMMA
    for b in blocks:
        fm, fz = oracle.bloch_f32(nodes32, T1, T2, np.zeros(N, np.float32), 1.0, np.float32(DEFAULT_GAMMA), b.rf,
                                  b.G, b.dt.astype(np.float32), mm, zz, history=False)
        mm, zz = (0 * fm).astype(np.complex64), fz
    assert fp64.rel_l2(m[:, 0], fm) < 2e-6
    assert fp64.rel_l2(z[:, 0], fz) < 1e-6
    # a 15-degree spoiled GRE approaches the Ernst steady state: |Mxy| ~ sin(15 deg) Mz-
    assert 0.05 < np.abs(m).mean() < np.sin(np.deg2rad(15.0))
    # complex FP64 k-space through the FP64 overload (every dense argument float64)
    traj = W.cartesian(res=(64, 64, 1), fov=(0.1, 0.1, 0.1))
    w = _lumped(mesh)
    assert w.dtype == np.float64 and abs(w.sum() - np.pi * 0.04 ** 2 * 0.08) / (np.pi * 0.04 ** 2 * 0.08) < 0.05
    M = sp.diags(w).tocsc()
    pts = [np.asarray(p, np.float64) for p in traj.points]
    t64 = np.asarray(traj.t, np.float64)
    Mxy = m.astype(np.complex128)
    K = Signal(0, M, pts, t64, mesh.nodes, np.zeros(N), np.asarray(T2, np.float64), Mxy, None)
    assert K.dtype == np.complex128 and K.shape == (64, 64, 1, 1)
    Ko = oracle.signal(M, *pts, t64, mesh.nodes, np.zeros(N), np.asarray(T2, np.float64), Mxy, dtype=np.float64,
                       threads=8)
    assert fp64.rel_l2(K, Ko) < 1e-12


def test_phase_contrast_config_full_size(cuda):
    import bench
    case = bench.build_case()
    N, traj, vel = case["N"], case["traj"], case["vel"]
    assert N >= 195_000 and traj.shape == (96, 96, 32)
    w = _lumped(case["mesh"], np.float32).astype(np.float32)
    M = sp.diags(w).tocsc()
    rng = np.random.default_rng(7)
    V = 4
    Mxy = ((rng.normal(size=(N, V)) + 1j * rng.normal(size=(N, V))) * 0.1).astype(np.complex64)
    r0 = case["mesh"].nodes.astype(np.float32)
    vel.update_timeshift(0.0)
    S = traj.n_samples
    pick = np.sort(rng.choice(S, 1000, replace=False))
    disp = np.stack([vel(float(t)) for t in signal_call_times(traj.t)[1:]])
    ref = fp64.signal(M, *traj.points, traj.t, r0, case["phi"], case["T2"], Mxy, disp=disp, pi_mode="float",
                      sample_idx=pick)
    for prec, tol in (("f32", 1e-5), ("bf16x3", 1e-4)):
        K = Signal(0, M, traj.points, traj.t, r0, case["phi"], case["T2"], Mxy, vel, precision=prec)
        err = fp64.rel_l2(K.reshape(S, V)[pick], ref)
        assert err < tol, (prec, err)


def test_precision_config_reduced_nodes(cuda):
    mesh = W.ellipsoid(40_000)
    N = mesh.n_nodes
    traj = W.radial3d(n_ro=256, n_spokes=256, kmax=500.0)
    assert np.abs(np.stack(traj.points)).max() <= 500.0 + 1e-3
    S, C = traj.n_samples, 8
    T1, T2 = W.tissue(N, 2)
    phi = W.off_resonance(N, 20.0, 2)
    coils = W.coil_maps(mesh.nodes, C, seed=3)
    pod = W.sinusoidal_pod(N, n_modes=10, amp=1e-3, period=800.0, n_frames=20, seed=2)
    pod.update_timeshift(120.0)
    w = _lumped(mesh, np.float32).astype(np.float32)
    M = sp.diags(w).tocsc()
    cols = (np.full(N, np.sin(np.deg2rad(15.0)), np.complex64)[:, None] * coils).astype(np.complex64)
    r0 = mesh.nodes.astype(np.float32)
    pick = np.sort(np.random.default_rng(3).choice(S, 512, replace=False))
    times = signal_call_times(traj.t)[1:]

    class _RunDisp:
        def __getitem__(self, g):
            return pod(float(times[g]))

    ref = fp64.signal(M, *traj.points, traj.t, r0, phi, T2, cols, disp=_RunDisp(), pi_mode="float", sample_idx=pick)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, cols, pod, precision="bf16x3")
    assert K.shape == (*traj.shape, C)
    err = fp64.rel_l2(K.reshape(S, C)[pick], ref)
    assert err < 1e-4, err


@pytest.mark.parametrize("precision,tol", [("f32", 1e-5), ("bf16x3", 2e-5)])
def test_node_partition_sums_to_whole_mesh(cuda, precision, tol):
    # the multi-GPU scheme (Phantom.py:194-239, MPIUtilities.py:13-26) through
    # the product path: each part's local lumped mass and Signal, summed as
    # gather_data does, equals the Signal of the whole mesh (parts run one
    # after another on this GPU; no collective is involved)
    from feelmri_b200.distributed import distribute_mesh
    mesh = W.tube(30_000, 0.012, 0.1)
    traj = W.cartesian(res=(16, 24, 8))
    rng = np.random.default_rng(4)
    N = mesh.n_nodes
    Mxy = ((rng.normal(size=(N, 2)) + 1j * rng.normal(size=(N, 2))) * 0.1).astype(np.complex64)
    phi = W.off_resonance(N, 20.0, 4)
    _, T2 = W.tissue(N, 4)
    vel = W.poiseuille_velocity(mesh.nodes, 0.012, v_max=1.0, period=60.0, n_frames=6)

    def signal(elems, nodes, l2g):
        w = _lumped(type(mesh)(nodes, elems), np.float32).astype(np.float32)
        term = vel.terms[0]
        from feelmri_b200.motion import SplineMotion, SplineTerm
        local = SplineMotion([SplineTerm(term.kind, term.coeffs, term.knots, modes=term.modes[l2g],
                                         period=term.period)])
        return Signal(0, sp.diags(w).tocsc(), traj.points, traj.t, nodes.astype(np.float32), phi[l2g], T2[l2g],
                      Mxy[l2g], local, precision=precision)

    whole = signal(mesh.elems, mesh.nodes, np.arange(N))
    total = np.zeros_like(whole)
    for rank in range(3):
        part = distribute_mesh(mesh.elems, mesh.nodes, 3, rank)
        total += signal(part.elems, part.nodes, part.local_to_global)
    assert fp64.rel_l2(total, whole) < tol
