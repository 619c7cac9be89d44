"""GPU Bloch sweep (solve_mri drop-in) against the FP32 restatement and FP64."""
import numpy as np
import pytest

import oracle
from oracle import fp64
from feelmri_b200 import workloads as W
from feelmri_b200.BlochSimulator import bloch_call_times, solve_mri

pytestmark = pytest.mark.gpu

GAMMA = np.float32(W.GAMMA)


def _setup(n=3000, seed=0):
    mesh = W.cylinder(n)
    N = mesh.n_nodes
    T1, T2 = W.tissue(N, seed)
    dB = np.random.default_rng(seed).normal(0, 1e-4, N).astype(np.float32)
    return mesh, N, T1, T2, dB


def _block():
    b = W.hard_pulse_block(0.0, 25.0, 5.0, grad=((3.0, -2.0, 1.0), 1.0, 2.0))
    return b


def test_static_history_matches_restatement(cuda):
    mesh, N, T1, T2, dB = _setup()
    b = _block()
    r0 = mesh.nodes.astype(np.float32)
    Mxy0 = np.zeros((N, 1), np.complex64)
    Mz0 = np.ones((N, 1), np.float32)
    mg, zg = solve_mri(r0, T1.reshape(-1, 1), T2.reshape(-1, 1), dB.reshape(-1, 1), 1.0, float(GAMMA),
                       b.rf.reshape(-1, 1), b.G, b.dt, np.abs(b.rf) != 0, Mxy0, Mz0, None)
    assert mg.shape == (N, b.rf.size) and mg.dtype == np.complex64 and mg.flags.f_contiguous
    assert zg.shape == (N, b.rf.size) and zg.dtype == np.float32
    mo, zo = oracle.bloch_f32(r0, T1, T2, dB, 1.0, GAMMA, b.rf, b.G, b.dt, Mxy0, Mz0)
    np.testing.assert_array_equal(mg[:, 0], Mxy0[:, 0])
    assert fp64.rel_l2(mg, mo) < 2e-6
    assert fp64.rel_l2(zg, zo) < 1e-6
    m64, z64 = fp64.bloch(r0, T1, T2, dB, 1.0, float(GAMMA), b.rf, b.G, b.dt, Mxy0, Mz0, history=True)
    # float32 vs float64: the reference's own single-precision error
    assert fp64.rel_l2(mg, m64) < 1e-5
    assert fp64.rel_l2(zg, z64) < 5e-6


def test_pod_motion_lowered_equals_sampled_callable(cuda):
    mesh, N, T1, T2, dB = _setup(2000)
    b = _block()
    r0 = mesh.nodes.astype(np.float32)
    pod = W.sinusoidal_pod(N, n_modes=5, amp=2e-3, period=4.0, n_frames=9)
    pod.update_timeshift(np.float32(0.75))
    args = (r0, T1, T2, dB, 1.0, float(GAMMA), b.rf, b.G, b.dt, np.abs(b.rf) != 0, np.zeros(N, np.complex64),
            np.ones(N, np.float32))
    m_low, z_low = solve_mri(*args, pod)

    calls = []

    def wrapped(t):  # a plain callable: not lowered, sampled at the reference's call times
        calls.append(t)
        return pod(t)

    m_tab, z_tab = solve_mri(*args, wrapped)
    np.testing.assert_array_equal(np.asarray(calls), bloch_call_times(b.dt))
    assert fp64.rel_l2(m_low, m_tab) < 1e-6
    disp = np.stack([pod(t) for t in bloch_call_times(b.dt)])
    mo, zo = oracle.bloch_f32(r0, T1, T2, dB, 1.0, GAMMA, b.rf, b.G, b.dt, np.zeros(N, np.complex64),
                              np.ones(N, np.float32), disp=disp)
    assert fp64.rel_l2(m_low, mo) < 2e-6
    assert fp64.rel_l2(z_low, zo) < 1e-6


@pytest.mark.parametrize("kind", ["spline_motion", "reference_classes"])
def test_velocity_pod_and_respiratory_sum(cuda, kind):
    import refmotion as R
    from feelmri_b200.motion import SplineMotion
    mesh, N, T1, T2, dB = _setup(1500)
    b = _block()
    r0 = mesh.nodes.astype(np.float32)
    vel = W.poiseuille_velocity(mesh.nodes, radius=0.04, period=3.0, n_frames=7)
    times = np.linspace(0, 6.0, 20)
    curve = 0.004 * np.sin(np.linspace(0, np.pi, 20))
    if kind == "spline_motion":
        motion = SplineMotion.rigid((0, 1, 0), times, curve, periodic=True) + vel
    else:
        # doubles of the reference's RespiratoryMotion + PODVelocity (a PODSum)
        from scipy.interpolate import PchipInterpolator
        fit = PchipInterpolator(times, curve)
        resp = R.respiratory_from_ppoly(fit.c, fit.x, np.array([0, 1, 0]), period=times[-1])
        term = vel.terms[0]
        motion = R.PODSum(resp, R.pod_from_ppoly(term.coeffs, term.knots, term.modes, velocity=True,
                                                 period=np.float32(term.period)))
    motion.update_timeshift(1.25)
    args = (r0, T1, T2, dB, 1.0, float(GAMMA), b.rf, b.G, b.dt, np.abs(b.rf) != 0, np.zeros(N, np.complex64),
            np.ones(N, np.float32))
    m_low, z_low = solve_mri(*args, motion)
    m_tab, z_tab = solve_mri(*args, lambda t: motion(t))
    assert fp64.rel_l2(m_low, m_tab) < 1e-6
    assert fp64.rel_l2(z_low, z_tab) < 1e-6


def test_dtype_dispatch_converts_like_pybind(cuda):
    mesh, N, T1, T2, dB = _setup(500)
    b = _block()
    r0 = mesh.nodes  # float64: converted to float32 in the second pass
    out64 = solve_mri(r0, T1.astype(np.float64), T2, dB, 1, GAMMA, b.rf.astype(np.complex128), b.G, b.dt,
                      np.abs(b.rf) != 0, np.zeros(N), np.ones(N), None)
    out32 = solve_mri(r0.astype(np.float32), T1, T2, dB, 1.0, float(GAMMA), b.rf, b.G, b.dt.astype(np.float32),
                      np.abs(b.rf) != 0, np.zeros(N, np.complex64), np.ones(N, np.float32), None)
    np.testing.assert_array_equal(out64[0], out32[0])
    with pytest.raises(TypeError):
        solve_mri(r0, T1, T2, dB, 1.0, GAMMA, b.rf, b.G, b.dt, None, np.zeros(N), np.ones(N), 3.0)
    with pytest.raises(ValueError):
        solve_mri(r0[:-1], T1, T2, dB, 1.0, GAMMA, b.rf, b.G, b.dt, np.abs(b.rf) != 0, np.zeros(N), np.ones(N), None)


def test_single_time_point_returns_initial_state(cuda):
    N = 10
    r0 = np.zeros((N, 3), np.float32)
    one = np.ones(N, np.float32)
    m, z = solve_mri(r0, one, one, 0 * one, 1.0, 1.0, np.zeros(1, np.complex64), np.zeros((1, 3), np.float32),
                     np.zeros(1, np.float32), np.zeros(1, bool), (0.5 + 0.5j) * one, 0.25 * one, None)
    np.testing.assert_array_equal(m[:, 0], (0.5 + 0.5j) * one)
    np.testing.assert_array_equal(z[:, 0], 0.25 * one)


def test_final_state_form_equals_history_last_column(cuda):
    import torch
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    mesh, N, T1, T2, dB = _setup(4000)
    b = _block()
    dev = torch.device("cuda")
    up = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
    inp = ops.BlochInputs(up(mesh.nodes.astype(np.float32), torch.float32), up(T1, torch.float32),
                          up(T2, torch.float32), up(dB, torch.float32), 1.0, float(GAMMA), up(b.rf, torch.complex64),
                          up(b.G, torch.float32), up(b.dt.astype(np.float32), torch.float32),
                          torch.zeros(N, dtype=torch.complex64, device=dev), torch.ones(N, device=dev))
    none = lower(None, N, dev)
    mh, zh = ops.bloch_solve(inp, none, history=True)
    mf, zf = ops.bloch_solve(inp, none, history=False)
    assert torch.equal(mh[-1], mf) and torch.equal(zh[-1], zf)
