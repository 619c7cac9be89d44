"""Drop-in for the reference module `feelmri.MRI`.

Signal keeps the reference's positional signature and overload order
(cpp/feelmri/MRI.h:43-83): float32 with a callable, float32 with None,
float64 with a callable, float64 with None.  The float64 overload is taken
only when every dense argument already is float64 / complex128 (the
no-conversion pass of pybind11); any other mix runs in float32.  The result is
a C-ordered (n_ro, n_lines, n_kz, V) complex array.

Keyword-only extension: precision="bf16x3" runs the split-BF16 tcgen05
tensor-core form on float32 inputs (precision=None keeps the drop-in choice).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _pybind as pb
from . import ops
from ._motion import lower, sample_table, table_motion

__all__ = ["Signal", "signal_call_times"]


def signal_call_times(t: np.ndarray) -> np.ndarray:
    """Times at which the reference calls pod_trajectory during one Signal:
    t(0,0,0) first (MRI.cpp:50), then once per run of equal consecutive times
    in (readout, line, kz) order (MRI.cpp:109-134)."""
    flat = np.ascontiguousarray(t).reshape(-1)
    if flat.size == 0:
        return np.zeros(0)
    starts = np.concatenate(([0], np.flatnonzero(flat[1:] != flat[:-1]) + 1))
    return np.concatenate(([flat[0]], flat[starts])).astype(np.float64)


def _load(args, T, convert: bool, want_none: bool):
    (rank, M, kloc, t, r0, phi, T2, Mxy, pod) = args
    C = np.complex64 if T == np.float32 else np.complex128
    return dict(
        rank=pb.py_int(rank, convert),
        M=pb.sparse_csc(M, T),
        kloc=pb.sequence_of(kloc, lambda k: pb.tensor(k, T, 3, convert)),
        t=pb.tensor(t, T, 3, convert),
        r0=pb.dense(r0, T, convert),
        phi=pb.dense(phi, T, convert, vector=True),
        T2=pb.dense(T2, T, convert, vector=True),
        Mxy=pb.dense(Mxy, C, convert),
        pod=pb.function_or_none(pod, want_none),
        T=T,
    )


def Signal(MPI_rank, M, kloc, t, r0, phi_dB0, T2, Mxy, pod_trajectory, *, precision: str | None = None):
    """Mass-weighted non-uniform DFT of the node magnetisation (see module docstring)."""
    args = (MPI_rank, M, kloc, t, r0, phi_dB0, T2, Mxy, pod_trajectory)
    for convert in (False, True):
        for T in (np.float32, np.float64):
            for want_none in (False, True):
                try:
                    a = _load(args, T, convert, want_none)
                except pb.NoMatch:
                    continue
                return _run(precision=precision, **a)
    raise pb.no_overload("Signal", args)


def _run(rank, M, kloc, t, r0, phi, T2, Mxy, pod, T, precision):
    if len(kloc) != 3:
        raise ValueError(f"Signal: kloc must hold (kx, ky, kz); got {len(kloc)} arrays")
    grid = kloc[0].shape
    for k in (*kloc[1:], t):
        if k.shape != grid:
            raise ValueError(f"Signal: k-space/time arrays differ in shape ({k.shape} vs {grid})")
    N = r0.shape[0]
    if r0.shape[1] != 3:
        raise ValueError(f"Signal: r0 must be (N, 3); got {r0.shape}")
    for name, arr in (("phi_dB0", phi), ("T2", T2)):
        if arr.shape[0] != N:
            raise ValueError(f"Signal: {name} has {arr.shape[0]} entries, r0 has {N} nodes")
    if Mxy.shape[0] != N:
        raise ValueError(f"Signal: Mxy has {Mxy.shape[0]} rows, r0 has {N} nodes")
    shape, indptr, indices, data = M
    if shape != (N, N):
        raise ValueError(f"Signal: M is {shape}, expected ({N}, {N})")
    prec = "f64" if T == np.float64 else "f32"
    if precision is not None:
        if precision == "bf16x3" and T == np.float64:
            raise TypeError("Signal: precision='bf16x3' takes float32 inputs")
        if precision not in ("bf16x3", prec):
            raise ValueError(f"Signal: precision={precision!r} does not match the {prec} inputs")
        prec = precision
    dev = ops.require_cuda()
    real = torch.float64 if T == np.float64 else torch.float32
    cplx = torch.complex128 if T == np.float64 else torch.complex64

    (d_indptr, d_indices, d_data, d_kx, d_ky, d_kz, d_t, d_r0, d_phi, d_T2, d_Mxy) = ops.upload_many(
        [(indptr, torch.int32), (indices, torch.int32), (data, real), (kloc[0], real), (kloc[1], real),
         (kloc[2], real), (t, real), (r0, real), (phi, real), (T2, real), (Mxy, cplx)], dev)
    inp = ops.SignalInputs(M=ops.SparseCSC(shape, d_indptr, d_indices, d_data), kx=d_kx, ky=d_ky, kz=d_kz, t=d_t,
                           r0=d_r0, phi=d_phi, T2=d_T2, Mxy=d_Mxy)
    motion = lower(pod, N, dev)
    if motion is None:
        calls = signal_call_times(t)
        table = sample_table(pod, calls, N, T, dev)
        motion = table_motion(table[1:].contiguous())  # the first call's result is unused
    out = ops.signal(inp, motion, prec)
    return ops.to_host(out)
