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
    """Rebuild the stored callables as feelmri_b200.Motion objects."""
    from feelmri_b200.Motion import POD, PODSum, PODVelocity, RespiratoryMotion, _periodic_fold
    from scipy.interpolate import PPoly

    def scalar(v, kind):
        v = float(v)
        return {"f32": np.float32(v), "f64": np.float64(v), "py": v, "none": None}[str(kind)]

    terms = []
    for k in range(int(d[f"{name}/n_terms"])):
        p = f"{name}/term{k}/"
        kind = str(d[p + "kind"])
        ts = scalar(d[p + "timeshift"], d[p + "timeshift_kind"])
        period = scalar(d[p + "period"], d[p + "period_kind"])
        if kind in ("POD", "PODVelocity"):
            obj = (PODVelocity if kind == "PODVelocity" else POD).__new__(PODVelocity if kind == "PODVelocity" else POD)
            obj._pp_batch = PPoly(d[p + "c"], d[p + "x"], extrapolate=bool(d[p + "extrapolate"]))
            obj._modes = np.ascontiguousarray(d[p + "modes"])
            obj.n_modes = obj._modes.shape[2]
            obj._weights = np.zeros(obj.n_modes, np.float32)
        else:
            obj = RespiratoryMotion.__new__(RespiratoryMotion)
            obj.interpolator = PPoly(d[p + "c"], d[p + "x"], extrapolate=bool(d[p + "extrapolate"]))
            obj.direction = d[p + "direction"]
        obj.timeshift = ts
        obj._period = period
        obj._fold_time = _periodic_fold(period)
        terms.append(obj)
    if len(terms) == 1:
        return terms[0]
    s = PODSum(terms[0], terms[1])
    s.timeshift = terms[0].timeshift
    return s


def test_motion_golden_host_classes_match_reference(cuda):
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


@pytest.mark.parametrize("dtype,tol", [(np.float32, 2e-4), (np.float64, 1e-9)])
def test_pod_construction_on_device(cuda, dtype, tol):
    # Motion.POD(backend="cuda"): the snapshot products on the GPU, the t x t
    # eigenproblem on the host; modes, weights and the evaluated motion match
    # the numpy construction (eigenvector signs are arbitrary: aligned first)
    from feelmri_b200.Motion import POD
    rng = np.random.default_rng(11)
    P, t, r_true = 6000, 24, 4
    times = np.linspace(0.0, 100.0, t)
    base = rng.normal(size=(P, 3, r_true))
    amp = np.array([3.0, 1.5, 0.7, 0.3])
    freq = np.arange(1, r_true + 1)  # distinct frequencies: a well-separated rank-4 history
    w = np.sin(2 * np.pi * freq[None, :] * times[:, None] / 100.0 + rng.uniform(0, 6, r_true)[None, :]) * amp
    data = (np.einsum("pcm,tm->pct", base, w) + 1e-4 * rng.normal(size=(P, 3, t))).astype(dtype)
    ref = POD(times, data, n_modes=3)
    dev = POD(times, data, n_modes=3, backend="cuda")
    assert dev.modes.dtype == ref.modes.dtype and dev.weights.dtype == ref.weights.dtype
    for m in range(3):
        s = np.sign(np.vdot(ref.modes[..., m].ravel(), dev.modes[..., m].ravel()))
        dm = dev.modes[..., m] * s
        dw = dev.weights[:, m] * s
        assert np.linalg.norm(dm - ref.modes[..., m]) / np.linalg.norm(ref.modes[..., m]) < tol
        assert np.linalg.norm(dw - ref.weights[:, m]) / np.linalg.norm(ref.weights[:, m]) < tol
    # the motion itself does not depend on the signs
    for tq in (0.0, 37.5, 99.0):
        a, b = ref(tq), dev(tq)
        assert np.linalg.norm(a - b) / np.linalg.norm(a) < tol
    # reproducible: FP64 sums in a fixed order
    again = POD(times, data, n_modes=3, backend="cuda")
    np.testing.assert_array_equal(again.modes, dev.modes)
