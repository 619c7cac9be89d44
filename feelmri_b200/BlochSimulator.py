"""Drop-in for the reference module `feelmri.BlochSimulator`.

solve_mri keeps the reference's positional signature, overloads and return
value (cpp/feelmri/BlochSimulator.h:50-80): two float32 overloads, chosen by
whether `pod_trajectory` is callable or None, with every array converted to
float32 / complex64 / bool by pybind11's rules.  It returns
(Mxy (N, n_t) complex64, Mz (N, n_t) float32), column 0 being the initial
state, both Fortran-ordered like the Eigen matrices the reference returns.
The sweep runs on the GPU (fm_bloch_solve_f32); motion callables from
feelmri.Motion are evaluated there too, any other callable is called at the
times the reference calls it (0.0, then the float32 running time of each
step) and its outputs are uploaded.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _pybind as pb
from . import ops
from ._motion import lower, sample_table, table_motion

__all__ = ["solve_mri", "bloch_call_times"]


def bloch_call_times(dt: np.ndarray) -> np.ndarray:
    """Times at which the reference calls pod_trajectory during one solve:
    0.0 first (BlochSimulator.cpp:44), then ti after each step, where ti
    accumulates dt[i+1] in float32 (BlochSimulator.cpp:67, :82-83)."""
    dt = np.asarray(dt, dtype=np.float32).reshape(-1)
    out = np.zeros(max(dt.size, 1), dtype=np.float64)
    if dt.size > 1:
        out[1:] = np.add.accumulate(dt[1:], dtype=np.float32).astype(np.float64)
    return out


def _load(args, convert: bool, want_none: bool):
    (r0, T1, T2, delta_B, M0, gamma, rf_all, G_all, dt, regime_idx, Mxy0, Mz0, pod) = args
    f32, c64 = np.float32, np.complex64
    return dict(
        r0=pb.dense(r0, f32, convert, cols=3),
        T1=pb.dense(T1, f32, convert, vector=True),
        T2=pb.dense(T2, f32, convert, vector=True),
        delta_B=pb.dense(delta_B, f32, convert, vector=True),
        M0=np.float32(pb.py_float(M0, convert)),
        gamma=np.float32(pb.py_float(gamma, convert)),
        rf=pb.dense(rf_all, c64, convert, vector=True),
        G=pb.dense(G_all, f32, convert, cols=3),
        dt=pb.dense(dt, f32, convert, vector=True),
        regime=pb.dense(regime_idx, np.bool_, convert, vector=True),
        Mxy0=pb.dense(Mxy0, c64, convert, vector=True),
        Mz0=pb.dense(Mz0, f32, convert, vector=True),
        pod=pb.function_or_none(pod, want_none),
    )


def solve_mri(r0, T1, T2, delta_B, M0, gamma, rf_all, G_all, dt, regime_idx, Mxy_initial, Mz_initial,
              pod_trajectory):
    """Bloch sweep of every node over every time step (see module docstring)."""
    args = (r0, T1, T2, delta_B, M0, gamma, rf_all, G_all, dt, regime_idx, Mxy_initial, Mz_initial,
            pod_trajectory)
    for convert in (False, True):
        for want_none in (False, True):
            try:
                a = _load(args, convert, want_none)
            except pb.NoMatch:
                continue
            return _run(**a)
    raise pb.no_overload("solve_mri", args)


def _run(r0, T1, T2, delta_B, M0, gamma, rf, G, dt, regime, Mxy0, Mz0, pod):
    N = r0.shape[0]
    n_t = rf.shape[0]
    for name, arr in (("T1", T1), ("T2", T2), ("delta_B", delta_B), ("Mxy_initial", Mxy0), ("Mz_initial", Mz0)):
        if arr.shape[0] != N:
            raise ValueError(f"solve_mri: {name} has {arr.shape[0]} entries, r0 has {N} nodes")
    for name, arr in (("G_all", G), ("dt", dt), ("regime_idx", regime)):
        if arr.shape[0] != n_t:
            raise ValueError(f"solve_mri: {name} has {arr.shape[0]} time points, rf_all has {n_t}")
    if n_t == 0:
        raise ValueError("solve_mri: rf_all is empty (the reference writes column 0 of an (N, 0) history)")
    dev = ops.require_cuda()

    def up(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dtype)

    inp = ops.BlochInputs(r0=up(r0, torch.float32), T1=up(T1, torch.float32), T2=up(T2, torch.float32),
                          delta_B=up(delta_B, torch.float32), M0=float(M0), gamma=float(gamma),
                          rf=up(rf, torch.complex64), G=up(G, torch.float32), dt=up(dt, torch.float32),
                          Mxy0=up(Mxy0, torch.complex64), Mz0=up(Mz0, torch.float32))
    motion = lower(pod, N, dev)
    if motion is None:
        table = sample_table(pod, bloch_call_times(dt), N, np.float32, dev)
        motion = table_motion(table)
    Mxy_h, Mz_h = ops.bloch_solve(inp, motion, history=True)
    # (n_t, N) row-major on the device == (N, n_t) column-major
    m, z = ops.to_host(Mxy_h, Mz_h)
    return m.T, z.T
