"""GPU Signal (MRI.Signal drop-in, FP32 and FP64 forms) against the oracle."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from oracle import fp64
from feelmri_b200 import workloads as W
from feelmri_b200.MRI import Signal, signal_call_times

pytestmark = pytest.mark.gpu


def _case(n=2500, V=3, seed=0, lumped=True):
    mesh = W.cylinder(n)
    N = mesh.n_nodes
    rng = np.random.default_rng(seed)
    Mxy = ((rng.normal(size=(N, V)) + 1j * rng.normal(size=(N, V))) * 0.1).astype(np.complex64)
    phi = W.off_resonance(N)
    _, T2 = W.tissue(N, seed)
    if lumped:
        M = sp.lil_matrix((N, N))
        M.setdiag(rng.uniform(1e-7, 3e-7, N))
    else:
        A = sp.random(N, N, density=8.0 / N, random_state=seed, format="csr")
        M = (A + A.T + sp.eye(N)).tocsc() * 1e-7
    return mesh, N, M, Mxy, phi, T2


def test_f32_static_matches_restatement_and_fp64(cuda):
    mesh, N, M, Mxy, phi, T2 = _case()
    traj = W.cartesian(res=(24, 20, 6))
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None)
    assert K.shape == (*traj.shape, 3) and K.dtype == np.complex64 and K.flags.c_contiguous
    Ko = oracle.signal(sp.csc_matrix(M), *traj.points, traj.t, r0, phi, T2, Mxy, dtype=np.float32)
    assert fp64.rel_l2(K, Ko) < 1e-5
    K64 = fp64.signal(sp.csc_matrix(M), *traj.points, traj.t, r0, phi, T2, Mxy, pi_mode="float")
    assert fp64.rel_l2(K, K64) < 1e-5


def test_f64_overload_only_when_everything_is_double(cuda):
    mesh, N, M, Mxy, phi, T2 = _case(n=1200, V=2)
    traj = W.cartesian(res=(12, 10, 4))
    d = np.float64
    pts = [p.astype(d) for p in traj.points]
    K = Signal(0, M, pts, traj.t.astype(d), mesh.nodes, phi.astype(d), T2.astype(d), Mxy.astype(np.complex128),
               None)
    assert K.dtype == np.complex128
    Ko = oracle.signal(sp.csc_matrix(M), *pts, traj.t.astype(d), mesh.nodes, phi, T2, Mxy, dtype=np.float64)
    assert fp64.rel_l2(K, Ko) < 1e-12
    K64 = fp64.signal(sp.csc_matrix(M), *pts, traj.t, mesh.nodes, phi, T2, Mxy.astype(np.complex128),
                      pi_mode="float")
    assert fp64.rel_l2(K, K64) < 1e-12
    # one float32 argument sends the whole call to the float32 overload
    Kmix = Signal(0, M, pts, traj.t.astype(d), mesh.nodes, phi, T2.astype(d), Mxy.astype(np.complex128), None)
    assert Kmix.dtype == np.complex64


def test_consistent_mass_and_split_node_ranges(cuda):
    mesh, N, M, Mxy, phi, T2 = _case(n=6000, V=1, lumped=False)
    traj = W.cartesian(res=(8, 4, 2))  # 64 samples: forces node splits over many blocks
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None)
    Ko = oracle.signal(sp.csc_matrix(M), *traj.points, traj.t, r0, phi, T2, Mxy, dtype=np.float32)
    assert fp64.rel_l2(K, Ko) < 1e-5
    K2 = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None)
    np.testing.assert_array_equal(K, K2)  # deterministic


def test_pod_motion_lowered_and_sampled(cuda):
    mesh, N, M, Mxy, phi, T2 = _case(n=2000, V=4)
    traj = W.cartesian(res=(16, 12, 4))
    r0 = mesh.nodes.astype(np.float32)
    vel = W.poiseuille_velocity(mesh.nodes, radius=0.04, period=50.0, n_frames=6)
    vel.update_timeshift(7.0)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, vel)
    calls = []

    def wrapped(t):
        calls.append(t)
        return vel(t)

    Kt = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, wrapped)
    np.testing.assert_array_equal(np.asarray(calls), signal_call_times(traj.t))
    assert fp64.rel_l2(K, Kt) < 1e-6
    disp = np.stack([vel(t) for t in signal_call_times(traj.t)[1:]])
    Ko = oracle.signal(sp.csc_matrix(M), *traj.points, traj.t, r0, phi, T2, Mxy, disp=disp, dtype=np.float32)
    assert fp64.rel_l2(K, Ko) < 1e-5


def test_runs_follow_sample_order_and_nan(cuda):
    mesh, N, M, Mxy, phi, T2 = _case(n=800, V=2)
    rng = np.random.default_rng(3)
    shape = (5, 7, 3)
    kx, ky, kz = (rng.uniform(-200, 200, shape).astype(np.float32) for _ in range(3))
    t = rng.choice(np.array([1.0, 2.0, 2.5], np.float32), size=shape)
    t[2, 3, 1] = np.nan
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, (kx, ky, kz), t, r0, phi, T2, Mxy, None)
    Ko = oracle.signal(sp.csc_matrix(M), kx, ky, kz, t, r0, phi, T2, Mxy, dtype=np.float32)
    finite = np.isfinite(Ko)
    assert np.array_equal(np.isfinite(K), finite)
    assert fp64.rel_l2(K[finite], Ko[finite]) < 1e-5


@pytest.mark.parametrize("V", [1, 2, 5, 8, 11])
def test_column_counts(cuda, V):
    mesh, N, M, Mxy, phi, T2 = _case(n=700, V=V)
    traj = W.radial3d(n_ro=16, n_spokes=40, kmax=300.0)
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None)
    Ko = oracle.signal(sp.csc_matrix(M), *traj.points, traj.t, r0, phi, T2, Mxy, dtype=np.float32)
    assert fp64.rel_l2(K, Ko) < 1e-5


def test_edge_cases(cuda):
    mesh, N, M, Mxy, phi, T2 = _case(n=300, V=2)
    r0 = mesh.nodes.astype(np.float32)
    z = np.zeros((0, 4, 2), np.float32)
    K = Signal(0, M, (z, z, z), z, r0, phi, T2, Mxy, None)
    assert K.shape == (0, 4, 2, 2)
    one = np.ones((1, 1, 1), np.float32) * 10.0
    K1 = Signal(0, M, (one, -one, one), one, r0, phi, T2, Mxy, None)
    Ko = oracle.signal(sp.csc_matrix(M), one, -one, one, one, r0, phi, T2, Mxy, dtype=np.float32)
    assert fp64.rel_l2(K1, Ko) < 1e-5
    with pytest.raises(ValueError):
        Signal(0, M, (one, one, one), one, r0[:-1], phi, T2, Mxy, None)
    with pytest.raises(TypeError):
        Signal(0.5, M, (one, one, one), one, r0, phi, T2, Mxy, None)
