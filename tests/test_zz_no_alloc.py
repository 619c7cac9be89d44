"""The no-allocation Bloch entry point against the workspace entry point.

fm_bloch_solve_f32_noalloc serves callers that may not allocate device
memory: its per-step scratch is a fixed array inside the library instead of
a workspace the caller allocates.  Both entry points are called here through
the C ABI on the same inputs, twice in a row with different inputs: first
with a 4-mode POD motion (the larger weights region), then without motion,
so that the previous call's contents are still in the shared array when the
second call runs.  Both entry points run the same kernels on the same inputs
and differ only in where the scratch lives, so the outputs must be equal bit
for bit.  This file is collected last so that a run stopping at
the first failure has run every other test; it also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

from feelmri_b200 import _lib as L
from feelmri_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _inputs(torch, dev, N, n_t, seed):
    rng = np.random.default_rng(seed)
    nodes = rng.uniform(-0.05, 0.05, (N, 3)).astype(np.float32)
    T1 = rng.uniform(800, 1200, N).astype(np.float32)
    T2 = rng.uniform(50, 100, N).astype(np.float32)
    dB = rng.normal(0, 1e-4, N).astype(np.float32)
    rf = np.zeros(n_t, np.complex64)
    rf[1:11] = 0.02 + 0.01j * seed
    G = np.zeros((n_t, 3), np.float32)
    G[20:60] = (3.0, -2.0, 1.0 + seed)
    dt = np.full(n_t, 0.01, np.float32)
    dt[40:] = 0.05
    up = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    return dict(r0=up(nodes), T1=up(T1), T2=up(T2), dB=up(dB), rf=up(rf), G=up(G), dt=up(dt),
                Mxy0=torch.zeros(N, dtype=torch.complex64, device=dev), Mz0=torch.ones(N, device=dev))


def _args(d, motion, N, n_t, hist_m, hist_z):
    a = L.BlochArgs()
    a.n_pos, a.n_time = N, n_t
    a.r0, a.T1, a.T2, a.delta_B = d["r0"].data_ptr(), d["T1"].data_ptr(), d["T2"].data_ptr(), d["dB"].data_ptr()
    a.M0, a.gamma = 1.0, float(np.float32(W.GAMMA))
    a.rf, a.G, a.dt = d["rf"].data_ptr(), d["G"].data_ptr(), d["dt"].data_ptr()
    a.Mxy0, a.Mz0 = d["Mxy0"].data_ptr(), d["Mz0"].data_ptr()
    a.motion = C.pointer(motion.struct)
    a.Mxy_hist, a.Mz_hist = hist_m.data_ptr(), hist_z.data_ptr()
    return a


def test_no_alloc_matches_workspace_entry_point_twice(cuda):
    import torch
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    lib = L.lib()
    dev = cuda
    torch.cuda.set_device(dev)
    ctx = ops.ctx_for(dev)
    N, n_t = 3000, 120
    for call, seed in enumerate((1, 2)):
        d = _inputs(torch, dev, N, n_t, seed)
        pod = W.sinusoidal_pod(N, n_modes=4, amp=1e-3, period=3.0, n_frames=6) if call == 0 else None
        motion = lower(pod, N, dev)
        ref_m = torch.empty((n_t, N), dtype=torch.complex64, device=dev)
        ref_z = torch.empty((n_t, N), dtype=torch.float32, device=dev)
        got_m = torch.full((n_t, N), float("nan"), dtype=torch.complex64, device=dev)
        got_z = torch.full((n_t, N), float("nan"), dtype=torch.float32, device=dev)
        a_ref = _args(d, motion, N, n_t, ref_m, ref_z)
        nbytes = C.c_size_t()
        L.check(lib.fm_bloch_workspace_size(C.byref(a_ref), C.byref(nbytes)))
        ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
        L.check(lib.fm_bloch_solve_f32(ctx, C.byref(a_ref), ws.data_ptr(), ws.numel()))
        a_new = _args(d, motion, N, n_t, got_m, got_z)
        L.check(lib.fm_bloch_solve_f32_noalloc(ctx, C.byref(a_new)))
        torch.cuda.synchronize(dev)
        rm, rz = ref_m.cpu().numpy(), ref_z.cpu().numpy()
        gm, gz = got_m.cpu().numpy(), got_z.cpu().numpy()
        assert np.all(np.isfinite(gm)) and np.all(np.isfinite(gz)), f"call {call}: outputs not written"
        assert np.array_equal(gm, rm), f"call {call}: Mxy differs from the workspace entry point"
        assert np.array_equal(gz, rz), f"call {call}: Mz differs from the workspace entry point"


def test_no_alloc_rejects_oversized_requests(cuda):
    import torch
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    lib = L.lib()
    dev = cuda
    N, n_t = 8, 200_000  # more steps than the fixed scratch holds
    d = _inputs(torch, dev, N, n_t, 1)
    m = torch.empty((n_t, N), dtype=torch.complex64, device=dev)
    z = torch.empty((n_t, N), dtype=torch.float32, device=dev)
    a = _args(d, lower(None, N, dev), N, n_t, m, z)
    status = lib.fm_bloch_solve_f32_noalloc(ops.ctx_for(dev), C.byref(a))
    assert status == L.FM_ERR_NOMEM
    assert "scratch" in L.last_error()
