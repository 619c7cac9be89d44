"""The oracle against analytic known answers (physics, not vectors from any
suite): hard-pulse flips, free precession, T1/T2 relaxation, a single-node
DFT, P1 lumping and the invariances of the mass-weighted sum."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from oracle import fp64
from feelmri_b200 import workloads as W
from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
from feelmri_b200.Assemble import tabulate_at_quadrature

GAMMA = W.GAMMA


def _nodes(n, seed=0):
    rng = np.random.default_rng(seed)
    return rng.uniform(-0.05, 0.05, (n, 3)).astype(np.float32)


@pytest.mark.parametrize("flip", [15.0, 30.0, 90.0])
def test_hard_pulse_on_resonance(flip):
    N = 4
    b = W.hard_pulse_block(0.0, flip, 0.1, rf_dur=0.1, dt_rf=0.01, dt=0.1)
    big = np.full(N, 1e12, np.float32)
    m, mz = oracle.bloch_f32(np.zeros((N, 3), np.float32), big, big, np.zeros(N, np.float32), 1.0, GAMMA, b.rf, b.G,
                             b.dt, np.zeros(N, np.complex64), np.ones(N, np.float32), history=False)
    th = np.deg2rad(flip)
    # rf along +x tips the magnetisation towards +y (the rotation's sign convention)
    np.testing.assert_allclose(m, 1j * np.sin(th), atol=2e-6)
    np.testing.assert_allclose(mz, np.cos(th), atol=2e-6)


def test_free_precession_and_relaxation():
    N = 16
    r0 = _nodes(N)
    T1 = np.full(N, 900.0, np.float32)
    T2 = np.full(N, 70.0, np.float32)
    dB = np.linspace(-1e-3, 1e-3, N).astype(np.float32)
    n_t = 51
    times = np.linspace(0, 10.0, n_t)
    G = np.tile(np.array([[5.0, -3.0, 2.0]], np.float32), (n_t, 1))
    rf = np.zeros(n_t, np.complex64)
    Mxy0 = (0.3 + 0.4j) * np.ones(N, np.complex64)
    Mz0 = np.full(N, 0.2, np.float32)
    m, mz = oracle.bloch_f32(r0, T1, T2, dB, 1.0, GAMMA, rf, G, np.diff(times, prepend=0), Mxy0, Mz0, history=False)
    t = times[-1]
    Bz = r0.astype(np.float64) @ G[0].astype(np.float64) + dB
    m_exp = Mxy0 * np.exp(-1j * GAMMA * Bz * t) * np.exp(-t / T2)
    mz_exp = 1.0 + (Mz0 - 1.0) * np.exp(-t / T1)
    # float32 accumulates ~1 ulp of a ~10 rad step angle per step
    np.testing.assert_allclose(m, m_exp, atol=2e-4)
    np.testing.assert_allclose(mz, mz_exp, atol=2e-6)
    m64, mz64 = fp64.bloch(r0, T1, T2, dB, 1.0, GAMMA, rf, G, np.diff(times, prepend=0), Mxy0, Mz0)
    np.testing.assert_allclose(m64, m_exp, atol=1e-10)
    np.testing.assert_allclose(mz64, mz_exp, atol=1e-12)


def test_bloch_float32_matches_float64():
    mesh = W.cylinder(500)
    N = mesh.n_nodes
    T1, T2 = W.tissue(N)
    blocks = W.spoiled_gre(3)
    b = blocks[0]
    r0 = mesh.nodes.astype(np.float32)
    dB = np.zeros(N, np.float32)
    m32, z32 = oracle.bloch_f32(r0, T1, T2, dB, 1.0, GAMMA, b.rf, b.G, b.dt, np.zeros(N, np.complex64),
                                np.ones(N, np.float32), history=True)
    m64, z64 = fp64.bloch(r0, T1, T2, dB, 1.0, GAMMA, b.rf, b.G, b.dt, np.zeros(N), np.ones(N), history=True)
    assert fp64.rel_l2(m32, m64) < 1e-5
    assert fp64.rel_l2(z32, z64) < 1e-6


def test_single_node_signal_closed_form():
    x = np.array([[0.013, -0.021, 0.007]], np.float64)
    w, m, phi, T2 = 0.37, 0.6 - 0.2j, 0.05, 80.0
    traj = W.cartesian(res=(8, 6, 2), fov=(0.1, 0.1, 0.1))
    M = sp.csc_matrix(np.array([[w]]))
    K = fp64.signal(M, traj.kx, traj.ky, traj.kz, traj.t, x, [phi], [T2], [[m]], pi_mode="exact")
    k = np.stack([traj.kx, traj.ky, traj.kz], -1).astype(np.float64)
    t = traj.t.astype(np.float64)
    expect = w * m * np.exp(-t / T2) * np.exp(1j * (phi * t - 2 * np.pi * (k @ x[0])))
    np.testing.assert_allclose(K[..., 0], expect, rtol=1e-12, atol=1e-15)
    K32 = oracle.signal(M, traj.kx, traj.ky, traj.kz, traj.t, x, [phi], [T2], [[m]], dtype=np.float32)
    assert fp64.rel_l2(K32[..., 0], expect) < 2e-6
    K64 = oracle.signal(M, traj.kx, traj.ky, traj.kz, traj.t, x, [phi], [T2], [[m]], dtype=np.float64,
                        pi_exact=True)
    assert fp64.rel_l2(K64[..., 0], expect) < 1e-13


def _signal_case(n=300, V=2, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-0.04, 0.04, (n, 3))
    Mxy = (rng.normal(size=(n, V)) + 1j * rng.normal(size=(n, V))).astype(np.complex64)
    phi = rng.normal(0, 0.1, n).astype(np.float32)
    T2 = rng.uniform(50, 100, n).astype(np.float32)
    M = sp.diags(rng.uniform(0.5, 1.5, n)).tocsc()
    return x, Mxy, phi, T2, M


def test_signal_node_permutation_and_partition_invariance():
    x, Mxy, phi, T2, M = _signal_case()
    traj = W.cartesian(res=(6, 5, 3))
    ref = fp64.signal(M, traj.kx, traj.ky, traj.kz, traj.t, x, phi, T2, Mxy)
    perm = np.random.default_rng(1).permutation(x.shape[0])
    Mp = M[perm][:, perm]
    alt = fp64.signal(Mp, traj.kx, traj.ky, traj.kz, traj.t, x[perm], phi[perm], T2[perm], Mxy[perm])
    assert fp64.rel_l2(alt, ref) < 1e-13
    # splitting the nodes over "ranks" and summing (gather_data) gives the same k-space
    parts = np.array_split(np.arange(x.shape[0]), 3)
    tot = sum(fp64.signal(M[p][:, p], traj.kx, traj.ky, traj.kz, traj.t, x[p], phi[p], T2[p], Mxy[p]) for p in parts)
    assert fp64.rel_l2(tot, ref) < 1e-13
    # the threaded C restatement sums node partitions the same way
    a = oracle.signal(M, traj.kx, traj.ky, traj.kz, traj.t, x, phi, T2, Mxy, dtype=np.float64, pi_exact=True,
                      threads=1)
    b = oracle.signal(M, traj.kx, traj.ky, traj.kz, traj.t, x, phi, T2, Mxy, dtype=np.float64, pi_exact=True,
                      threads=4)
    assert fp64.rel_l2(a, ref) < 1e-12
    assert fp64.rel_l2(b, ref) < 1e-12


def test_signal_float_pi_is_what_the_reference_uses():
    x, Mxy, phi, T2, M = _signal_case(n=50, V=1)
    traj = W.cartesian(res=(4, 4, 2))
    a = oracle.signal(M, traj.kx, traj.ky, traj.kz, traj.t, x, phi, T2, Mxy, dtype=np.float64, pi_exact=False)
    b = fp64.signal(M, traj.kx, traj.ky, traj.kz, traj.t, x, phi, T2, Mxy, pi_mode="float")
    assert fp64.rel_l2(a, b) < 1e-12


def test_p1_lumped_mass_is_quarter_volume():
    mesh = W.cylinder(2000)
    fe, qr = FiniteElement(dtype=np.float64), QuadratureRule(order=2, dtype=np.float64)
    qw, tab = tabulate_at_quadrature(fe, qr, np.float64)
    indptr, indices, data = oracle.mass_csc(mesh.elems, mesh.nodes, qw, tab)
    lumped = oracle.csc_rowsum(indptr, indices, data)
    exact = fp64.lumped_p1(mesh.elems, mesh.nodes)
    np.testing.assert_allclose(lumped, exact, rtol=1e-12)
    X = mesh.nodes[mesh.elems]
    vol = np.abs(np.linalg.det(X[:, 1:] - X[:, :1])).sum() / 6
    assert abs(lumped.sum() - vol) < 1e-12 * vol
    # consistent P1 mass: diagonal 2 * vol / 20 and off-diagonal vol / 20 per element
    M = sp.csc_matrix((data, indices, indptr), shape=(mesh.n_nodes,) * 2)
    assert abs(M.sum() - vol) < 1e-12 * vol
    assert np.all(np.diff(indices[indptr[0]:indptr[1]]) > 0)


def test_float32_quadrature_offsets_lumping_by_float_rounding():
    mesh = W.cylinder(1000)
    fe, qr = FiniteElement(), QuadratureRule(order=2)  # float32 as the reference's wrappers
    qw, tab = tabulate_at_quadrature(fe, qr, np.float64)
    indptr, indices, data = oracle.mass_csc(mesh.elems, mesh.nodes, qw, tab)
    lumped = oracle.csc_rowsum(indptr, indices, data)
    exact = fp64.lumped_p1(mesh.elems, mesh.nodes)
    err = np.max(np.abs(lumped / exact - 1))
    assert 0 < err < 1e-6
