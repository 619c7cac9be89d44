"""Batched split-BF16 Signal: problems of uneven node and sample counts, run
kinds, column counts and motions share one persistent tensor-core launch.
Each problem's k-space is bit-identical to the same problem run alone (same
tuning) and within 1e-4 relative L2 of the FP64 oracle."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from oracle import fp64
from feelmri_b200 import ops, workloads as W
from feelmri_b200._motion import lower
from feelmri_b200.MRI import signal_call_times

pytestmark = pytest.mark.gpu

TOL = 1e-4  # split-BF16 form against FP64


def _problem(cuda, mesh, traj, V, seed, motion=None):
    N = mesh.n_nodes
    rng = np.random.default_rng(seed)
    Mxy = ((rng.normal(size=(N, V)) + 1j * rng.normal(size=(N, V))) * 0.1).astype(np.complex64)
    phi = W.off_resonance(N, 20.0, seed)
    _, T2 = W.tissue(N, seed)
    w = rng.uniform(1e-7, 3e-7, N).astype(np.float32)
    up = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(cuda, dt)  # noqa: E731
    M = ops.SparseCSC((N, N), up(np.arange(N + 1, dtype=np.int32), torch.int32),
                      up(np.arange(N, dtype=np.int32), torch.int32), up(w))
    r0 = mesh.nodes.astype(np.float32)
    inp = ops.SignalInputs(M=M, kx=up(traj.kx), ky=up(traj.ky), kz=up(traj.kz), t=up(traj.t), r0=up(r0),
                           phi=up(phi), T2=up(T2), Mxy=up(Mxy, torch.complex64))
    host = dict(M=sp.diags(w.astype(np.float64)).tocsc(), traj=traj, r0=r0, phi=phi, T2=T2, Mxy=Mxy, pod=motion)
    return inp, lower(motion, N, cuda), host


def _oracle(h, idx):
    disp = None
    if h["pod"] is not None:
        disp = np.stack([h["pod"](t) for t in signal_call_times(h["traj"].t)[1:]])
    return fp64.signal(h["M"], *h["traj"].points, h["traj"].t, h["r0"], h["phi"], h["T2"], h["Mxy"], disp=disp,
                       pi_mode="float", sample_idx=idx)


def _batch(cuda):
    vel_mesh = W.tube(6000, 0.012, 0.1)
    vel = W.poiseuille_velocity(vel_mesh.nodes, 0.012, v_max=1.0, period=60.0, n_frames=6)
    vel.update_timeshift(7.0)
    specs = [
        (W.cylinder(2500), W.cartesian(res=(8, 24, 16)), 1, None),
        (vel_mesh, W.cartesian(res=(10, 32, 12)), 4, vel),
        (W.ellipsoid(9000, (0.03, 0.025, 0.02)), W.spiral_stack(n_ro=48, n_interleaves=6, n_kz=8), 2, None),
        (W.cylinder(4000), W.radial3d(n_ro=10, n_spokes=200, kmax=300.0), 9, None),
        (W.cylinder(1500), W.cartesian(res=(6, 8, 40)), 3, None),
    ]
    return [_problem(cuda, m, t, V, 10 + i, mo) for i, (m, t, V, mo) in enumerate(specs)]


@pytest.mark.parametrize("tuning", [ops.Tuning(split_nodes=2048), ops.Tuning(split_nodes=0, kz_cap=8)])
def test_batch_equals_alone_and_oracle(cuda, tuning):
    probs = _batch(cuda)
    outs = [torch.empty((*inp.kx.shape, inp.Mxy.shape[1]), dtype=torch.complex64, device=cuda) for inp, _, _ in probs]
    batch = ops.SignalBatch([(inp, mo, o) for (inp, mo, _), o in zip(probs, outs)], tuning)
    batch.run()
    for (inp, mo, h), o in zip(probs, outs):
        alone = torch.empty_like(o)
        ops.SignalBatch([(inp, mo, alone)], tuning).run()
        got = o.cpu().numpy()
        # the same problem alone: identical bits (its units and sums do not depend on the batch)
        np.testing.assert_array_equal(got, alone.cpu().numpy())
        S = got.size // got.shape[-1]
        idx = np.random.default_rng(0).choice(S, min(S, 400), replace=False)
        err = fp64.rel_l2(got.reshape(S, -1)[idx], _oracle(h, idx))
        assert err < TOL, err


def test_batch_matches_single_call_form(cuda):
    probs = _batch(cuda)[:3]
    outs = ops.signal_batch([(inp, mo, None) for inp, mo, _ in probs], ops.Tuning(split_nodes=4096))
    for (inp, mo, _), o in zip(probs, outs):
        single = ops.signal(inp, mo, "bf16x3")
        # different node splits group the FP32 sums differently; each form is
        # about 5e-6 from FP64, so the two agree to 1e-5
        assert fp64.rel_l2(o.cpu().numpy(), single.cpu().numpy()) < 1e-5


def test_batch_with_empty_problem(cuda):
    probs = _batch(cuda)[:2]
    mesh = W.cylinder(2000)
    traj = W.cartesian(res=(4, 8, 4))
    inp, mo, _ = _problem(cuda, mesh, traj, 2, 3)
    empty = ops.SignalInputs(M=ops.SparseCSC((0, 0), inp.M.indptr[:1], inp.M.indices[:0], inp.M.data[:0]),
                             kx=inp.kx, ky=inp.ky, kz=inp.kz, t=inp.t, r0=inp.r0[:0], phi=inp.phi[:0],
                             T2=inp.T2[:0], Mxy=inp.Mxy[:0])
    outs = ops.signal_batch([(p[0], p[1], None) for p in probs] + [(empty, lower(None, 0, cuda), None)],
                            ops.Tuning(split_nodes=2048))
    assert torch.count_nonzero(outs[-1]).item() == 0
    assert all(torch.isfinite(torch.view_as_real(o)).all().item() for o in outs)


def test_node_staging_paths_agree(cuda):
    # node blocks are staged by bulk copies when the inputs are 16-byte
    # aligned and by register loads otherwise; both give the same bits
    inp, mo, _ = _batch(cuda)[1]
    N = inp.r0.shape[0]
    def shifted(t):
        flat = t.reshape(-1)
        buf = torch.empty(flat.numel() + 1, dtype=t.dtype, device=cuda)
        buf[1:].copy_(flat)
        return buf[1:].view(t.shape)  # 4 bytes past an aligned address
    odd = ops.SignalInputs(M=inp.M, kx=inp.kx, ky=inp.ky, kz=inp.kz, t=inp.t, r0=shifted(inp.r0),
                           phi=shifted(inp.phi), T2=shifted(inp.T2), Mxy=inp.Mxy)
    assert odd.r0.data_ptr() % 16 != 0 and odd.r0.shape == (N, 3)
    tune = ops.Tuning(split_nodes=2048)
    a = ops.signal_batch([(inp, mo, None)], tune)[0]
    b = ops.signal_batch([(odd, mo, None)], tune)[0]
    np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
