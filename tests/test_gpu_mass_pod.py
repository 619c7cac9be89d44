"""GPU mass assembly / lumping and POD tensordot / motion evaluation against
the oracle and the golden vectors of the reference's Motion.py."""
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from oracle import fp64
from feelmri_b200 import workloads as W
from feelmri_b200.Assemble import MassAssemble, mass_lumped, tabulate_at_quadrature
from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
from feelmri_b200.POD import tensordot_modes_weights

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "motion_golden.npz"


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_mass_assembly_sparsity_exact_values_close(cuda, dtype):
    mesh = W.cylinder(6000)
    fe, qr = FiniteElement(), QuadratureRule(order=2)
    nodes = mesh.nodes.astype(dtype)
    M = MassAssemble(mesh.elems, nodes, fe, qr)
    assert isinstance(M, sp.csc_matrix) and M.dtype == dtype and M.shape == (mesh.n_nodes,) * 2
    qw, tab = tabulate_at_quadrature(fe, qr, dtype)
    indptr, indices, data = oracle.mass_csc(mesh.elems, nodes, qw, tab)
    np.testing.assert_array_equal(M.indptr, indptr)
    np.testing.assert_array_equal(M.indices, indices)
    tol = 1e-12 if dtype == np.float64 else 2e-6
    np.testing.assert_allclose(M.data, data, rtol=tol, atol=0)
    lump = mass_lumped(mesh.elems, nodes, fe, qr)
    ref = oracle.csc_rowsum(indptr, indices, data)
    np.testing.assert_allclose(lump, ref, rtol=tol, atol=0)
    # the reference's lumping of the GPU matrix (scipy on the CSC) agrees bit for bit
    np.testing.assert_array_equal(lump, np.asarray(M.sum(axis=1)).ravel())


def test_mass_overloads_follow_pybind(cuda):
    mesh = W.cylinder(300)
    fe, qr = FiniteElement(), QuadratureRule(order=2)
    assert MassAssemble(mesh.elems, mesh.nodes, fe, qr).dtype == np.float64
    # int64 connectivity needs conversion, and the second pass picks float
    assert MassAssemble(mesh.elems.astype(np.int64), mesh.nodes, fe, qr).dtype == np.float32


def test_lumped_sum_is_volume(cuda):
    mesh = W.ellipsoid(20000)
    fe, qr = FiniteElement(dtype=np.float64), QuadratureRule(order=2, dtype=np.float64)
    lump = mass_lumped(mesh.elems, mesh.nodes, fe, qr)
    np.testing.assert_allclose(lump, fp64.lumped_p1(mesh.elems, mesh.nodes), rtol=1e-12)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tensordot(cuda, dtype):
    rng = np.random.default_rng(0)
    modes = rng.normal(size=(5000, 3, 10)).astype(dtype)
    w = rng.normal(size=10).astype(dtype)
    out = tensordot_modes_weights(modes, w)
    ref = np.einsum("pcm,m->pc", modes.astype(np.float64), w.astype(np.float64))
    np.testing.assert_allclose(out, ref, rtol=1e-5 if dtype == np.float32 else 1e-13, atol=1e-5)
    with pytest.raises(TypeError):
        tensordot_modes_weights(modes, w.astype(np.float64 if dtype == np.float32 else np.float32))
    with pytest.raises(TypeError):
        tensordot_modes_weights(np.asfortranarray(modes), w)


def _golden_objects(d, name):
    """Rebuild the stored callables as doubles of the reference's classes."""
    import refmotion as R

    def scalar(v, kind):
        v = float(v)
        return {"f32": np.float32(v), "f64": np.float64(v), "py": v, "none": None}[str(kind)]

    terms = []
    for k in range(int(d[f"{name}/n_terms"])):
        p = f"{name}/term{k}/"
        kind = str(d[p + "kind"])
        ts = scalar(d[p + "timeshift"], d[p + "timeshift_kind"])
        period = scalar(d[p + "period"], d[p + "period_kind"])
        extrapolate = bool(d[p + "extrapolate"])
        if kind in ("POD", "PODVelocity"):
            obj = R.pod_from_ppoly(d[p + "c"], d[p + "x"], d[p + "modes"], velocity=kind == "PODVelocity",
                                   extrapolate=extrapolate, timeshift=ts, period=period)
        else:
            obj = R.respiratory_from_ppoly(d[p + "c"], d[p + "x"], d[p + "direction"], extrapolate=extrapolate,
                                           timeshift=ts, period=period)
        terms.append(obj)
    if len(terms) == 1:
        return terms[0]
    s = R.PODSum(terms[0], terms[1])
    s.timeshift = terms[0].timeshift
    return s


def test_motion_golden_doubles_match_reference(cuda):
    # the test doubles reproduce the reference's own outputs (so the device
    # comparisons below compare against the reference, not against the doubles)
    d = np.load(GOLDEN)
    for name in d["cases"]:
        obj = _golden_objects(d, name)
        gold = d[f"{name}/out"]
        for i, t in enumerate(d[f"{name}/t"]):
            y = np.broadcast_to(np.asarray(obj(float(t))), gold[i].shape)
            # the modes x weights GEMV may sum in another order: float32 rounding
            # of the largest terms bounds the difference
            scale = np.nanmax(np.abs(gold)) if np.isfinite(gold).any() else 1.0
            np.testing.assert_allclose(y, gold[i], rtol=1e-5, atol=2e-7 * scale, equal_nan=True,
                                       err_msg=f"{name} t={t}")


def test_motion_golden_device_weights_bit_exact(cuda):
    """Device fold + PPoly + float32 cast (+ velocity scaling) reproduce the
    reference's float32 weights exactly: modes are unit vectors so that each
    node's displacement equals one weight."""
    import torch
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    d = np.load(GOLDEN)
    dev = torch.device("cuda")
    for name in d["cases"]:
        obj = _golden_objects(d, name)
        if hasattr(obj, "pod1"):
            continue
        t = d[f"{name}/t"]
        gold_w = d[f"{name}/weights"]
        if hasattr(obj, "_modes"):
            r = obj._modes.shape[2]
            eye = np.zeros((r, 3, r), np.float32)
            eye[np.arange(r), 0, np.arange(r)] = 1.0
            obj._modes = eye
            low = lower(obj, r, dev)
            disp = ops.motion_eval(low, r, t, dev).cpu().numpy()
            got = disp[:, :, 0]
            np.testing.assert_array_equal(got, gold_w, err_msg=name)
        else:
            low = lower(obj, 1, dev)
            disp = ops.motion_eval(low, 1, t, dev).cpu().numpy()[:, 0, :]
            np.testing.assert_array_equal(disp, d[f"{name}/out"][:, 0, :], err_msg=name)


def test_motion_golden_device_displacements(cuda):
    import torch
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    d = np.load(GOLDEN)
    dev = torch.device("cuda")
    for name in d["cases"]:
        obj = _golden_objects(d, name)
        gold = d[f"{name}/out"]
        low = lower(obj, gold.shape[1], dev)
        assert low is not None, name
        disp = ops.motion_eval(low, gold.shape[1], d[f"{name}/t"], dev).cpu().numpy()
        scale = np.nanmax(np.abs(gold)) if np.isfinite(gold).any() else 1.0
        np.testing.assert_allclose(disp, gold, rtol=1e-5, atol=2e-7 * scale, equal_nan=True, err_msg=name)


def _numpy_snapshot_pod(times, data, n_modes):
    # the method of snapshots in plain numpy: eigenpairs of X^T X, the
    # n_modes largest, modes X e / sqrt(lambda), coefficients X^T modes
    X = data.reshape(-1, times.shape[0])
    lam, vec = np.linalg.eigh(X.T @ X)
    keep = np.argsort(lam)[::-1][:n_modes]
    phi = X @ (vec[:, keep] / np.sqrt(lam[keep]))
    return phi.reshape(data.shape[0], -1, n_modes), X.T @ phi


@pytest.mark.parametrize("dtype,tol", [(np.float32, 2e-4), (np.float64, 1e-9)])
def test_pod_construction_on_device(cuda, dtype, tol):
    # snapshot_pod: the snapshot products on the GPU, the t x t eigenproblem
    # on the host; modes and weights match the numpy construction
    # (eigenvector signs are arbitrary: aligned first), and so does the
    # motion built from them
    from feelmri_b200.motion import SplineMotion, calculate_pod_on_device, snapshot_pod
    rng = np.random.default_rng(11)
    P, t, r_true = 6000, 24, 4
    times = np.linspace(0.0, 100.0, t)
    base = rng.normal(size=(P, 3, r_true))
    amp = np.array([3.0, 1.5, 0.7, 0.3])
    freq = np.arange(1, r_true + 1)  # distinct frequencies: a well-separated rank-4 history
    w = np.sin(2 * np.pi * freq[None, :] * times[:, None] / 100.0 + rng.uniform(0, 6, r_true)[None, :]) * amp
    data = (np.einsum("pcm,tm->pct", base, w) + 1e-4 * rng.normal(size=(P, 3, t))).astype(dtype)
    ref_modes, ref_w = _numpy_snapshot_pod(times, data, 3)
    modes, weights = snapshot_pod(times, data, 3)
    assert modes.dtype == dtype and weights.dtype == dtype and modes.shape == (P, 3, 3)
    signs = []
    for m in range(3):
        s = np.sign(np.vdot(ref_modes[..., m].ravel(), modes[..., m].ravel()))
        signs.append(s)
        assert np.linalg.norm(modes[..., m] * s - ref_modes[..., m]) / np.linalg.norm(ref_modes[..., m]) < tol
        assert np.linalg.norm(weights[:, m] * s - ref_w[:, m]) / np.linalg.norm(ref_w[:, m]) < tol
    # the motion itself does not depend on the signs
    a = SplineMotion.from_samples(ref_modes.astype(np.float32), times, ref_w, periodic=False)
    b = SplineMotion.from_samples(modes.astype(np.float32), times, weights, periodic=False)
    for tq in (0.0, 37.5, 99.0):
        assert np.linalg.norm(a(tq) - b(tq)) / np.linalg.norm(a(tq)) < max(tol, 1e-5)
    # reproducible: FP64 sums in a fixed order
    again, _ = snapshot_pod(times, data, 3)
    np.testing.assert_array_equal(again, modes)

    # the hook that replaces a POD-like object's calculate_pod keeps the local nodes
    class _PodLike:
        pass
    pl = _PodLike()
    pl.times, pl.data, pl.n_modes = times, data, 3
    pl.local_to_global_map = np.arange(0, P, 7)
    hm, hw = calculate_pod_on_device(pl)
    np.testing.assert_array_equal(hm, modes[pl.local_to_global_map])
    np.testing.assert_array_equal(hw, weights)
