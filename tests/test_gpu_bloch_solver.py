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


def _small_case():
    mesh = W.cylinder(2000)
    N = mesh.n_nodes
    T1, T2 = W.tissue(N)
    return mesh.nodes.astype(np.float32), N, T1, T2, _blocks()[:4]


def test_scalar_and_array_parameters_agree(cuda):
    # scalars are filled on the device, arrays uploaded: same bits either way
    nodes, N, _, _, blocks = _small_case()
    a = BlochSolver(blocks, nodes, M0=1.0, T1=900.0, T2=80.0, delta_B=0.0, gamma=W.GAMMA)
    b = BlochSolver(blocks, nodes, M0=1.0, T1=np.full(N, 900.0, np.float32), T2=np.full((N, 1), 80.0),
                    delta_B=np.zeros(N), gamma=W.GAMMA, initial_Mxy=np.zeros(N), initial_Mz=np.ones(N))
    ma, za = a.solve()
    mb, zb = b.solve()
    np.testing.assert_array_equal(ma, mb)
    np.testing.assert_array_equal(za, zb)
    # host views keep the reference's construction: (N, 1) arrays
    assert a.T1.shape == (N, 1) and a.T1.dtype == np.float32 and a.initial_Mxy.dtype == np.complex64
    np.testing.assert_array_equal(a.initial_Mxy, b.initial_Mxy)


def test_state_arrays_follow_the_reference(cuda):
    # a held initial_Mz is updated in place by each solve; an in-place edit of
    # initial_Mxy is what the next solve starts from (Bloch.py:363-368)
    nodes, N, T1, T2, blocks = _small_case()
    s = BlochSolver(blocks, nodes, M0=1.0, T1=T1, T2=T2, gamma=W.GAMMA)
    held = s.initial_Mz
    s.solve()
    fresh = BlochSolver(blocks, nodes, M0=1.0, T1=T1, T2=T2, gamma=W.GAMMA)
    fresh.solve()
    np.testing.assert_array_equal(held, fresh.initial_Mz)   # written back in place
    edit = (np.random.default_rng(3).normal(size=N) * 0.1).astype(np.complex64)
    s.initial_Mxy[:, 0] = edit
    m1, z1 = s.solve(start=-1)
    t = BlochSolver(blocks, nodes, M0=1.0, T1=T1, T2=T2, gamma=W.GAMMA, initial_Mxy=edit,
                    initial_Mz=fresh.initial_Mz[:, 0].copy())
    m2, z2 = t.solve(start=-1)
    np.testing.assert_array_equal(m1, m2)
    np.testing.assert_array_equal(z1, z2)


def _mixed_blocks():
    """Blocks of different lengths, dt changes, empty gaps and stored states."""
    blocks = []
    t = 0.0
    for i in range(5):
        b = W.hard_pulse_block(t, 15.0 + 5 * i, 3.0 + i, grad=((1.0, -2.0, 0.5), 0.4, 0.8),
                               store=(i in (1, 4)), dt=0.05 if i % 2 else 0.1)
        blocks.append(b)
        t += 3.0 + i
        gap = W.hard_pulse_block(t, 0.0, 1.5)
        gap.empty = True
        gap.store_magnetization = (i == 2)
        blocks.append(gap)
        t += 1.5
    return blocks


@pytest.mark.parametrize("motion", ["none", "pod", "pod_sum"])
def test_sequence_sweep_equals_block_loop(cuda, motion):
    # the whole sequence in one launch (fm_bloch_sequence_f32) against the
    # per-block solves with the state carried between them: same bits
    mesh = W.cylinder(3000)
    N = mesh.n_nodes
    T1, T2 = W.tissue(N)
    nodes = mesh.nodes.astype(np.float32)
    dB = np.random.default_rng(2).normal(0, 1e-4, N).astype(np.float32)

    def make_pod():
        if motion == "none":
            return None
        p = W.sinusoidal_pod(N, n_modes=3, amp=1e-3, period=9.0, n_frames=7)
        if motion == "pod_sum":
            p = p + W.sinusoidal_pod(N, n_modes=2, amp=5e-4, period=5.0, n_frames=5, seed=9)
        return p

    results = []
    for path in ("sequence", "blocks"):
        s = BlochSolver(_mixed_blocks(), nodes, M0=1.0, T1=T1, T2=T2, delta_B=dB, gamma=W.GAMMA,
                        pod_trajectory=make_pod())
        if path == "blocks":
            s._solve_sequence = s._solve_blocks
        m, z = s.solve()
        results.append((m, z, s.initial_Mxy.copy(), s.initial_Mz.copy()))
    for a, b in zip(*results):
        np.testing.assert_array_equal(a, b)
    assert results[0][0].shape == (N, 3)


class _Quantity:
    """Just enough of a pint quantity: a magnitude in one unit."""
    _TO = {("ms", "ms"): 1.0, ("s", "ms"): 1e3, ("rad*Hz/T", "rad/ms/mT"): 1e-6}

    def __init__(self, m, units):
        self.m, self.units = m, units

    def m_as(self, units):
        return self.m * self._TO[(self.units, units)]

    def __add__(self, other):
        return _Quantity(self.m + other.m_as(self.units), self.units)


class _RefBlock:
    """A block with the reference SequenceBlock interface (Bloch.py:17-141):
    _discretization() as a quantity in ms, __call__(times) -> (rf, (Gm, Gp, Gs)),
    time_extent, empty, store_magnetization."""

    def __init__(self, block):
        self._b = block
        self.empty = block.empty
        self.store_magnetization = block.store_magnetization
        self.time_extent = [_Quantity(float(block.times[0]), "ms"), _Quantity(float(block.times[-1]), "ms")]

    def _discretization(self):
        return _Quantity(np.asarray(self._b.times, np.float64), "ms")

    def __call__(self, t):
        idx = np.searchsorted(self._b.times, t)
        return self._b.rf[idx], tuple(self._b.G[idx, d] for d in range(3))


class _RefSequence:
    def __init__(self, blocks):
        self.blocks = blocks
        self.Nb_blocks = len(blocks)


class _RefPhantom:
    def __init__(self, nodes):
        self.local_nodes = nodes


class _RefScanner:
    gamma = _Quantity(42.58e6 * 2 * np.pi, "rad*Hz/T")


@pytest.mark.parametrize("with_motion", [False, True])
def test_reference_signature_drop_in(cuda, with_motion):
    # BlochSolver(sequence, phantom, scanner, M0, T1, T2, delta_B,
    # pod_trajectory, initial_Mxy, initial_Mz) as unchanged reference scripts
    # build it (Bloch.py:276-297), with pint-like T1/T2 in seconds: the one-
    # launch sweep equals the per-block loop bit for bit and the reference's
    # block loop restated on the oracle within FP32 tolerance
    mesh = W.cylinder(2500)
    N = mesh.n_nodes
    T1, T2 = W.tissue(N)
    nodes = mesh.nodes.astype(np.float32)
    dB = np.random.default_rng(5).normal(0, 1e-4, (N, 1)).astype(np.float32)
    plain = _mixed_blocks()
    seq = _RefSequence([_RefBlock(b) for b in plain])

    def make(pod):
        return BlochSolver(seq, _RefPhantom(nodes), _RefScanner(), 1.0, _Quantity(T1.reshape(-1, 1) / 1e3, "s"),
                           _Quantity(T2.reshape(-1, 1) / 1e3, "s"), dB, pod, 0.0, None)

    pods = [W.sinusoidal_pod(N, n_modes=3, amp=1e-3, period=9.0, n_frames=7) if with_motion else None
            for _ in range(3)]
    one = make(pods[0])
    assert one.gamma == pytest.approx(W.GAMMA, rel=1e-12)
    m1, z1 = one.solve()
    loop = make(pods[1])
    loop._solve_sequence = loop._solve_blocks
    m2, z2 = loop.solve()
    np.testing.assert_array_equal(m1, m2)
    np.testing.assert_array_equal(z1, z2)
    np.testing.assert_array_equal(one.initial_Mxy, loop.initial_Mxy)
    # the oracle gets the T1, T2 the solver received: seconds converted to ms
    T1ms = _Quantity(T1.reshape(-1, 1) / 1e3, "s").m_as("ms").reshape(-1)
    T2ms = _Quantity(T2.reshape(-1, 1) / 1e3, "s").m_as("ms").reshape(-1)
    rm, rz, _, _ = _reference_loop(plain, nodes, T1ms, T2ms, dB.reshape(-1), pods[2], np.zeros(N, np.complex64),
                                   np.ones(N, np.float32))
    # ten blocks of FP32 steps: the libm sin/cos of the GPU and of the host
    # differ by an ulp here and there, which the recovery terms carry on
    assert fp64.rel_l2(m1, rm) < 2e-6
    assert fp64.rel_l2(z1, rz) < 2e-6
    # the reference reads the blocks at solve time: a block appended later is seen
    seq.blocks.append(_RefBlock(plain[1]))
    assert len(one.blocks) == len(plain) + 1
