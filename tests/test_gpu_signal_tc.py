"""Split-BF16 tensor-core Signal (precision="bf16x3") against the FP64
oracle: at most 1e-4 relative L2 on factored Cartesian runs and on generic
(non-separable) runs, with motion, several column counts and tile edges."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import fp64
from feelmri_b200 import workloads as W
from feelmri_b200.MRI import Signal, signal_call_times

pytestmark = pytest.mark.gpu

TOL = 1e-4  # split-BF16 form against FP64


def _case(n=3000, V=4, seed=0):
    mesh = W.cylinder(n)
    N = mesh.n_nodes
    rng = np.random.default_rng(seed)
    Mxy = ((rng.normal(size=(N, V)) + 1j * rng.normal(size=(N, V))) * 0.1).astype(np.complex64)
    phi = W.off_resonance(N)
    _, T2 = W.tissue(N, seed)
    M = sp.lil_matrix((N, N))
    M.setdiag(rng.uniform(1e-7, 3e-7, N))
    return mesh, N, M, Mxy, phi, T2


def _ref(M, traj, r0, phi, T2, Mxy, pod=None, idx=None):
    disp = None
    if pod is not None:
        disp = np.stack([pod(t) for t in signal_call_times(traj.t)[1:]])
    return fp64.signal(sp.csc_matrix(M), *traj.points, traj.t, r0, phi, T2, Mxy, disp=disp, pi_mode="float",
                       sample_idx=idx)


def test_factored_cartesian_static(cuda):
    mesh, N, M, Mxy, phi, T2 = _case()
    traj = W.cartesian(res=(12, 24, 8))
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    assert K.dtype == np.complex64 and K.shape == (*traj.shape, 4)
    err = fp64.rel_l2(K, _ref(M, traj, r0, phi, T2, Mxy))
    assert err < TOL, err


def test_factored_cartesian_with_flow(cuda):
    mesh, N, M, Mxy, phi, T2 = _case(n=5000)
    traj = W.cartesian(res=(16, 40, 32), fov=(0.1, 0.1, 0.1))
    r0 = mesh.nodes.astype(np.float32)
    vel = W.poiseuille_velocity(mesh.nodes, radius=0.04, period=60.0, n_frames=6)
    vel.update_timeshift(11.0)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, vel, precision="bf16x3")
    err = fp64.rel_l2(K, _ref(M, traj, r0, phi, T2, Mxy, pod=vel))
    assert err < TOL, err
    K32 = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, vel)
    assert fp64.rel_l2(K, K32) < TOL


def test_generic_radial_runs(cuda):
    mesh, N, M, Mxy, phi, T2 = _case(n=2500, V=8)
    traj = W.radial3d(n_ro=12, n_spokes=300, kmax=500.0)
    r0 = mesh.nodes.astype(np.float32)
    pod = W.sinusoidal_pod(N, n_modes=3, amp=1e-3, period=50.0, n_frames=8)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, pod, precision="bf16x3")
    err = fp64.rel_l2(K, _ref(M, traj, r0, phi, T2, Mxy, pod=pod))
    assert err < TOL, err


@pytest.mark.parametrize("V", [1, 3, 17])
def test_column_groups_and_tiles(cuda, V):
    mesh, N, M, Mxy, phi, T2 = _case(n=1500, V=V)
    traj = W.cartesian(res=(4, 140, 6))  # 140 lines: two row tiles
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    err = fp64.rel_l2(K, _ref(M, traj, r0, phi, T2, Mxy))
    assert err < TOL, err


def test_many_kz_columns_and_spiral(cuda):
    mesh, N, M, Mxy, phi, T2 = _case(n=1200, V=4)
    traj = W.cartesian(res=(3, 8, 70))  # 70 kz values: several column tiles
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    assert fp64.rel_l2(K, _ref(M, traj, r0, phi, T2, Mxy)) < TOL
    sp_traj = W.spiral_stack(n_ro=64, n_interleaves=4, n_kz=4)
    K = Signal(0, M, sp_traj.points, sp_traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    assert fp64.rel_l2(K, _ref(M, sp_traj, r0, phi, T2, Mxy)) < TOL


def test_deterministic_and_edge_cases(cuda):
    mesh, N, M, Mxy, phi, T2 = _case(n=800, V=2)
    traj = W.cartesian(res=(5, 6, 3))
    r0 = mesh.nodes.astype(np.float32)
    a = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    b = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    np.testing.assert_array_equal(a, b)
    t = traj.t.copy()
    t[1, 2, 1] = np.nan
    K = Signal(0, M, traj.points, t, r0, phi, T2, Mxy, None, precision="bf16x3")
    bad = ~np.isfinite(K)
    assert bad[1, 2, 1].all()
    with pytest.raises(TypeError):
        d = np.float64
        Signal(0, M, [p.astype(d) for p in traj.points], traj.t.astype(d), mesh.nodes, phi.astype(d), T2.astype(d),
               Mxy.astype(np.complex128), None, precision="bf16x3")


@pytest.mark.parametrize("res,V", [((4, 140, 6), 17), ((6, 96, 32), 4), ((3, 64, 16), 8)])
def test_repeat_calls_identical(cuda, res, V):
    """Several units per block and several column groups: repeated calls give
    the same bits (the block's warps hand over node blocks, phase tables and
    stages through barriers only, and the split sums are reduced in a fixed
    order)."""
    mesh, N, M, Mxy, phi, T2 = _case(n=1500, V=V)
    traj = W.cartesian(res=res)
    r0 = mesh.nodes.astype(np.float32)
    first = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    for _ in range(3):
        np.testing.assert_array_equal(Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3"),
                                      first)


def test_deep_node_sums_stay_accurate(cuda):
    """Tens of thousands of nodes per sample: the tensor core's truncating FP32
    accumulation must not grow with the node count (accumulators are drained
    into round-to-nearest sums every 512 nodes)."""
    mesh = W.tube(60_000, 0.012, 0.1)
    N = mesh.n_nodes
    rng = np.random.default_rng(5)
    Mxy = ((rng.normal(size=(N, 4)) + 1j * rng.normal(size=(N, 4))) * 0.2).astype(np.complex64)
    M = sp.diags(np.full(N, 2.3e-10)).tocsc()
    phi = W.off_resonance(N)
    _, T2 = W.tissue(N)
    traj = W.cartesian(res=(4, 96, 32), fov=(0.1, 0.1, 0.1))
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    idx = np.random.default_rng(0).choice(traj.n_samples, 400, replace=False)
    ref = _ref(M, traj, r0, phi, T2, Mxy, idx=idx)
    err = fp64.rel_l2(K.reshape(-1, 4)[idx], ref)
    assert err < 3e-5, err


def test_stacked_small_slabs(cuda):
    # static positions and equal kz offsets in every run: runs of 8 lines x 8 kz
    # are stacked several per unit; each run's block must come out alone
    mesh, N, M, Mxy, phi, T2 = _case(n=4000, V=2, seed=5)
    traj = W.spiral_stack(n_ro=40, n_interleaves=8, n_kz=8)
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    err = fp64.rel_l2(K, _ref(M, traj, r0, phi, T2, Mxy))
    assert err < TOL, err
    K32 = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None)
    assert fp64.rel_l2(K, K32) < TOL


@pytest.mark.parametrize("n_lines", [77, 140])
def test_stacked_lines_across_runs(cuda, n_lines):
    # slabs whose line count does not divide the 128 rows of a unit (77) or
    # exceeds them (140): units take 128 consecutive lines of the runs laid
    # end to end, so a unit starts inside one run and ends inside another;
    # every sample must come out once, with its own run's decay
    mesh, N, M, Mxy, phi, T2 = _case(n=3000, V=2, seed=8)
    traj = W.cartesian(res=(7, n_lines, 8))
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    idx = np.random.default_rng(9).choice(traj.n_samples, 1500, replace=False)
    err = fp64.rel_l2(K.reshape(traj.n_samples, -1)[idx], _ref(M, traj, r0, phi, T2, Mxy, idx=idx))
    assert err < TOL, err
    K32 = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None)
    assert fp64.rel_l2(K, K32) < TOL


def test_unstackable_runs_fall_back(cuda):
    # kz offsets that change from run to run: the stacking check must refuse
    mesh, N, M, Mxy, phi, T2 = _case(n=3000, V=1, seed=6)
    traj = W.cartesian(res=(10, 12, 8))
    kz = traj.kz * (1.0 + 0.01 * np.arange(10, dtype=np.float32)[:, None, None])
    traj = W.Trajectory(traj.kx, traj.ky, kz.astype(np.float32), traj.t)
    r0 = mesh.nodes.astype(np.float32)
    K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
    err = fp64.rel_l2(K, _ref(M, traj, r0, phi, T2, Mxy))
    assert err < TOL, err


@pytest.mark.parametrize("scale", [1.0, 1.0e8])
def test_phase_range_is_checked(cuda, scale):
    # the tensor-core form reduces k . r modulo one cycle in fixed point, which
    # holds for (|kx|+|ky|+|kz|)(|x|+|y|+|z|) below 2^27 cycles: in range the
    # result matches FP64, beyond it the call fails instead of returning wrong
    # samples (|kx|+|ky|+|kz| up to ~140 1/m here; nodes scaled to ~1e7 m are
    # far out of range)
    from feelmri_b200._lib import FeelMRIError
    mesh, N, M, Mxy, phi, T2 = _case(n=2000, V=1)
    traj = W.cartesian(res=(8, 16, 4))
    r0 = (mesh.nodes * scale).astype(np.float32)
    if scale == 1.0:
        K = Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
        assert fp64.rel_l2(K, _ref(M, traj, r0, phi, T2, Mxy)) < TOL
    else:
        with pytest.raises(FeelMRIError, match="2\\^27"):
            Signal(0, M, traj.points, traj.t, r0, phi, T2, Mxy, None, precision="bf16x3")
        # the context is still usable
        K = Signal(0, M, traj.points, traj.t, mesh.nodes.astype(np.float32), phi, T2, Mxy, None, precision="bf16x3")
        assert np.isfinite(K).all()


def test_staged_mode_rows_match_global_reads(cuda):
    """A POD term of several modes: the tensor-core form stages each node
    block's mode rows in shared memory with the block's other inputs.  The
    same call with the modes at an address that is not 16-byte aligned reads
    them from global memory instead; both agree bit for bit, and with FP64."""
    import torch
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    mesh, N, M, Mxy, phi, T2 = _case(n=6000, V=8, seed=3)
    traj = W.radial3d(n_ro=16, n_spokes=96, kmax=500.0)
    r0 = mesh.nodes.astype(np.float32)
    pod = W.sinusoidal_pod(N, n_modes=10, amp=1e-3, period=50.0, n_frames=8, seed=4)
    dev = torch.device("cuda", 0)
    up = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)
    Mc = sp.csc_matrix(M)
    inp = ops.SignalInputs(M=ops.SparseCSC(Mc.shape, up(Mc.indptr, torch.int32), up(Mc.indices, torch.int32),
                                           up(Mc.data)),
                           kx=up(traj.kx), ky=up(traj.ky), kz=up(traj.kz), t=up(traj.t), r0=up(r0), phi=up(phi),
                           T2=up(T2), Mxy=up(Mxy, torch.complex64))
    aligned = lower(pod, N, dev)
    assert aligned.struct.terms[0].modes % 16 == 0 and aligned.struct.terms[0].n_modes == 10
    K_staged = ops.signal(inp, aligned, "bf16x3").cpu().numpy()
    shifted = lower(pod, N, dev)
    rows = torch.empty(N * 30 + 1, dtype=torch.float32, device=dev)[1:]
    rows.copy_(torch.from_numpy(np.ascontiguousarray(pod.terms[0].modes, np.float32).reshape(-1)).to(dev))
    shifted.struct.terms[0].modes = rows.data_ptr()
    shifted.keep.append(rows)
    K_global = ops.signal(inp, shifted, "bf16x3").cpu().numpy()
    np.testing.assert_array_equal(K_staged.view(np.uint64), K_global.view(np.uint64))
    err = fp64.rel_l2(K_staged.reshape(*traj.shape, 8), _ref(M, traj, r0, phi, T2, Mxy, pod=pod))
    assert err < TOL, err
