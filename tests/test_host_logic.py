"""Host-side logic that needs no GPU: the autotuner's shape classes and cache
file, the serving loop's footprint and latency statistics, the SPAMM block's
physics (through the FP64 oracle) and the batching workload generator."""
import json

import numpy as np
import torch

from oracle import fp64
from feelmri_b200 import autotune, ops, workloads as W
from feelmri_b200.serving import Request, footprint_bytes, latency_stats


def _fake_problem(N, grid, V):
    z = lambda *s: torch.zeros(*s)  # noqa: E731
    inp = ops.SignalInputs(M=None, kx=z(grid), ky=z(grid), kz=z(grid), t=z(grid), r0=z(N, 3), phi=z(N), T2=z(N),
                           Mxy=torch.zeros(N, V, dtype=torch.complex64))
    return (inp, None, None)


def test_shape_class_buckets():
    a = [_fake_problem(10_000, (8, 16, 8), 2), _fake_problem(20_000, (8, 16, 8), 1)]
    b = [_fake_problem(10_500, (8, 16, 8), 2), _fake_problem(19_000, (8, 16, 8), 1)]
    c = [_fake_problem(10_000, (8, 16, 8), 4), _fake_problem(20_000, (8, 16, 8), 1)]
    assert autotune.shape_class(a) == autotune.shape_class(b)  # same log2 buckets
    assert autotune.shape_class(a) != autotune.shape_class(c)  # wider columns
    assert autotune.shape_class(a) != autotune.shape_class(a[:1])


def test_tuning_cache_file_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "tuning.json"
    monkeypatch.setenv("FEELMRI_B200_TUNING", str(path))
    monkeypatch.setattr(autotune, "_cache", {})
    probs = [_fake_problem(50_000, (32, 32, 16), 2)]
    key = autotune.shape_class(probs)
    autotune._cache[key] = ops.Tuning(split_nodes=8192, kz_cap=16)
    autotune._store()
    assert json.loads(path.read_text())[key] == {"split_nodes": 8192, "kz_cap": 16}
    monkeypatch.setattr(autotune, "_cache", {})
    assert autotune.cached(probs) == ops.Tuning(split_nodes=8192, kz_cap=16)
    # a cached batch class is returned without timing anything
    tuning, tried = autotune.tune(probs)
    assert tuning == ops.Tuning(split_nodes=8192, kz_cap=16) and tried == {}


def test_candidates_are_valid_tunings():
    assert len(set(autotune.CANDIDATES)) == len(autotune.CANDIDATES)
    for t in autotune.CANDIDATES:
        s = t.struct()
        assert s.split_nodes == t.split_nodes >= 0 and s.kz_cap == t.kz_cap >= 0


def test_latency_stats_and_footprint():
    st = latency_stats([0.1, 0.2, 0.3, 0.4])
    assert st["n"] == 4 and abs(st["p50_s"] - 0.25) < 1e-12 and st["p99_s"] <= 0.4 + 1e-12
    assert latency_stats([])["n"] == 0
    mesh = W.cylinder(2000)
    N = mesh.n_nodes
    T1, T2 = W.tissue(N, 0)

    def req(traj, coils):
        return Request(rid=0, mesh=mesh, T1=T1, T2=T2, phi=np.zeros(N, np.float32), blocks=[], traj=traj,
                       coils=np.ones((N, coils), np.complex64))
    small = footprint_bytes(req(W.cartesian(res=(8, 8, 8)), 1))
    big = footprint_bytes(req(W.cartesian(res=(32, 32, 8)), 4))
    assert 0 < small < big


def test_spamm_block_tags_mz():
    b = W.spamm_block(0.0, tag_spacing=0.008, tail=0.1)
    x = np.linspace(-0.02, 0.02, 81)
    r0 = np.stack([x, np.zeros_like(x), np.zeros_like(x)], 1).astype(np.float32)
    N = x.size
    slow = np.full(N, 1e9, np.float32)  # no relaxation
    res = fp64.bloch(r0, slow, slow, np.zeros(N, np.float32), 1.0, W.GAMMA, b.rf, b.G, b.dt.astype(np.float32),
                     np.zeros(N, np.complex64), np.ones(N, np.float32))
    Mz = np.asarray(res[1] if isinstance(res, tuple) else res).reshape(N, -1)[:, -1]
    ke = 2 * np.pi / 0.008
    np.testing.assert_allclose(Mz, -np.cos(ke * x), atol=1e-5)


def test_batching_workload_is_seeded_and_in_range():
    import bench
    a = bench.build_batch_requests_host(6)
    b = bench.build_batch_requests_host(6)
    assert [r.n_nodes for r in a] == [r.n_nodes for r in b]
    for r in a:
        assert 4_000 <= r.n_nodes <= 320_000
        assert 1 <= r.n_coils <= 2
        assert r.traj.shape[2] >= 8  # every trajectory is a kz stack (factorable slabs)
        assert r.weights.shape == (r.n_nodes,) and abs(r.weights.sum() / r.weights.sum()) == 1
        assert 4_000 <= r.traj.n_samples <= 210_000


def test_cpu_sample_counts_what_it_runs():
    # the bounded CPU step of the reference arm: a fraction of nodes for Bloch
    # and of readout rows for Signal, units = sum of nodes x sampled samples
    import bench
    reqs = bench.build_batch_requests_host(2)
    units, sec, det = bench.cpu_step(reqs, 0.01, 2)
    want = sum(r.n_nodes * r.traj.kx[:max(1, int(np.ceil(0.01 * r.traj.shape[0])))].size for r in reqs)
    assert units == want and sec > 0 and det["bloch_s"] >= 0 and det["signal_s"] > 0
    info = bench.cpu_info()
    assert info["threads_usable"] >= 1 and info["logical_cpus"] >= 1


def _csc_arrays(m, dtype):
    import scipy.sparse as sp
    c = sp.csc_matrix(m)
    return c.shape, c.indptr.astype(np.int32), c.indices.astype(np.int32), c.data.astype(dtype)


def test_lil_conversion_matches_scipy():
    # the Signal caster converts a float lil_matrix natively; the arrays must be
    # exactly those of scipy.sparse.csc_matrix(lil) with the data force-cast
    import scipy.sparse as sp
    from feelmri_b200 import _hostconv, _pybind as pb
    rng = np.random.default_rng(7)
    cases = []
    N = 5000
    D = sp.lil_matrix((N, N), dtype=np.float64)
    D.setdiag(rng.uniform(1e-7, 3e-7, N))
    cases.append(D)                                               # the lumped mass: a diagonal
    for seed, dt in ((1, np.float64), (2, np.float32)):
        R = sp.random(700, 400, density=0.02, random_state=seed, format="lil", dtype=dt)
        R[3, :] = 0                                               # an empty row
        cases.append(R)                                           # general pattern: the scatter path
    P = sp.lil_matrix((6, 4), dtype=np.float64)
    P[0, 2], P[1, 0], P[5, 3] = 1.0, -2.0, 3.0                    # not monotone in row order
    cases.append(P)
    cases.append(sp.lil_matrix((0, 0)))
    cases.append(sp.lil_matrix((5, 3)))
    for m in cases:
        for T in (np.float32, np.float64):
            got = pb.sparse_csc(m, T)
            want = _csc_arrays(m, T)
            assert got[0] == want[0]
            for g, w in zip(got[1:], want[1:]):
                assert g.dtype == w.dtype
                np.testing.assert_array_equal(g, w)
        for threads in (1, 3):
            r = _hostconv.lil_to_csc(m.rows, m.data, m.shape[0], m.shape[1], threads)
            c = sp.csc_matrix(m)
            np.testing.assert_array_equal(r[0], c.indptr)
            np.testing.assert_array_equal(r[1], c.indices)
            np.testing.assert_array_equal(r[2], c.data.astype(np.float64))


def test_lil_conversion_declines_what_scipy_must_handle():
    import scipy.sparse as sp
    from feelmri_b200 import _hostconv, _pybind as pb
    m = sp.lil_matrix((4, 4), dtype=np.float64)
    m[1, 2] = 5.0
    rows = m.rows.copy()
    rows[0] = [3]                                                 # lists of unequal length
    assert _hostconv.lil_to_csc(rows, m.data, 4, 4) is None
    rows = m.rows.copy()
    rows[1] = [9]
    assert _hostconv.lil_to_csc(rows, m.data, 4, 4) is None       # column index >= n_cols
    data = m.data.copy()
    data[1] = ["x"]
    assert _hostconv.lil_to_csc(m.rows, data, 4, 4) is None       # a value that is not a number
    # complex lil goes through scipy and the caster's real-part cast
    z = sp.lil_matrix((3, 3), dtype=np.complex128)
    z[0, 0] = 1 + 2j
    got = pb.sparse_csc(z, np.float32)
    np.testing.assert_array_equal(got[3], np.array([1.0], np.float32))


def test_term_timeshifts_follow_the_lowering():
    # the block-sequence sweep reads each block's timeshifts without lowering
    # again; they must be exactly what lower() would put in the descriptor
    from feelmri_b200._motion import lower, term_timeshifts
    import refmotion as R
    N = 50
    rng = np.random.default_rng(0)

    def pod(r, n_t):
        return R.pod_from_samples(rng.normal(size=(N, 3, r)).astype(np.float32), np.linspace(0.0, 10.0, n_t),
                                  rng.normal(size=(n_t, r)))
    a, b, c = pod(2, 5), pod(1, 5), pod(3, 6)
    s1 = W.sinusoidal_pod(N, n_modes=2, n_frames=5)
    s2 = W.sinusoidal_pod(N, n_modes=1, n_frames=5, seed=3)
    for obj in (a, R.PODSum(a, b), R.PODSum(R.PODSum(a, b), c), s1, s1 + s2):
        for t0 in (0.0, np.float32(2.5), np.float64(7.25), 3):
            obj.update_timeshift(t0)
            low = lower(obj, N, torch.device("cpu"))
            got = term_timeshifts(obj)
            want = [(low.struct.terms[k].timeshift, low.struct.terms[k].timeshift_kind)
                    for k in range(low.struct.n_terms)]
            assert got == want


def test_recon_grid_and_analytic_weights():
    # voxel centres on the DFT-centred grid; path-Jacobian density weights
    # (readout speed times in-plane radius, scaled to mean 1)
    from feelmri_b200 import Recon
    X, Y, Z = Recon.grid_points((4, 5, 1), (0.08, 0.1, 0.01))
    np.testing.assert_allclose(X[:, 0, 0], np.array([-2, -1, 0, 1]) * 0.02, atol=1e-7)
    np.testing.assert_allclose(Y[0, :, 0], np.array([-2, -1, 0, 1, 2]) * 0.02, atol=1e-7)
    assert np.all(Z == 0)
    # a 2-D radial spoke pair: uniform speed, so the weight is the radius
    r = np.linspace(-1.0, 1.0, 9)
    ang = np.array([0.3, 1.9])
    kx = (r[:, None] * np.cos(ang)[None, :])[..., None]
    ky = (r[:, None] * np.sin(ang)[None, :])[..., None]
    w = Recon.dcf_path_jacobian(kx, ky).reshape(kx.shape)
    want = np.abs(r)[:, None, None] * np.ones_like(kx)
    np.testing.assert_allclose(w, want / want.mean(), rtol=1e-6)
    # parallel lines (power 0): the weight follows the readout speed only
    kx = np.cumsum(np.array([1.0, 1.0, 2.0, 2.0, 1.0]))[:, None, None] * np.ones((1, 3, 2))
    w = Recon.dcf_path_jacobian(kx, np.zeros_like(kx), radial_power=0).reshape(kx.shape)
    speed = np.gradient(kx, axis=0)
    np.testing.assert_allclose(w, speed / speed.mean(), rtol=1e-6)


def test_spline_motion_host_evaluation():
    # SplineMotion's host evaluation against scipy's PPoly on the same
    # coefficients: float64 spline at the shifted, folded time rounded to
    # float32, velocity scaling by float32(t), float32 contraction; NaN
    # outside the knots without a period; a sum adds the terms
    from scipy.interpolate import PPoly
    from feelmri_b200.motion import SplineMotion
    rng = np.random.default_rng(3)
    N, r = 40, 3
    modes = rng.normal(size=(N, 3, r)).astype(np.float32)
    times = np.linspace(0.0, 8.0, 9)
    samples = rng.normal(size=(9, r))
    m = SplineMotion.from_samples(modes, times, samples, periodic=True)
    v = SplineMotion.from_samples(modes, times, samples, periodic=False, velocity=True)
    pp = PPoly(m.terms[0].coeffs, m.terms[0].knots, extrapolate=False)
    for ts in (0.0, 1.5):
        m.update_timeshift(ts)
        v.update_timeshift(ts)
        for t in (0.0, 0.3, 7.999, 8.0, 13.25):
            tau = (t + ts) - 8.0 * np.floor((t + ts) / 8.0)
            w = pp(tau).astype(np.float32)
            np.testing.assert_array_equal(m.terms[0].coefficients_at(tau), w)
            np.testing.assert_allclose(m(t), np.einsum("ncr,r->nc", modes, w), rtol=1e-6, atol=1e-6)
            raw = pp(t + ts)
            if np.all(np.isfinite(raw)):
                np.testing.assert_allclose(v(t), np.einsum("ncr,r->nc", modes, raw.astype(np.float32) *
                                                           np.float32(t)), rtol=1e-6, atol=1e-6)
            else:
                assert np.all(np.isnan(v(t)))
    both = m + v
    both.update_timeshift(0.5)
    m.update_timeshift(0.5)
    v.update_timeshift(0.5)
    np.testing.assert_array_equal(both(2.0), (m(2.0) + v(2.0)).astype(np.float32))
    rigid = SplineMotion.rigid((0, 2, 0), times, np.sin(times), periodic=False)
    assert rigid(1.0).shape == (1, 3) and rigid(1.0)[0, 0] == 0 and rigid(1.0)[0, 2] == 0


def test_install_as_feelmri_patches_reference_modules(tmp_path):
    # a stand-in reference package: install_as_feelmri must route the native
    # modules to the drop-ins and replace BlochSolver (and, on request,
    # POD.calculate_pod) whether feelmri.Bloch is imported before or after
    import importlib
    import sys
    import feelmri_b200
    from feelmri_b200.Bloch import BlochSolver
    from feelmri_b200.motion import calculate_pod_on_device
    pkg = tmp_path / "feelmri"
    pkg.mkdir()
    (pkg / "__init__.py").write_text("")
    (pkg / "Bloch.py").write_text("from feelmri.BlochSimulator import solve_mri\nclass BlochSolver:\n    pass\n")
    (pkg / "Motion.py").write_text("class POD:\n    def calculate_pod(self, remove_mean=False):\n"
                                   "        return 'host'\n")
    saved = {k: v for k, v in sys.modules.items() if k == "feelmri" or k.startswith("feelmri.")}
    sys.path.insert(0, str(tmp_path))
    try:
        for k in saved:
            del sys.modules[k]
        feelmri_b200.install_as_feelmri(device_pod=True)
        bloch = importlib.import_module("feelmri.Bloch")  # imported after the install
        assert bloch.BlochSolver is BlochSolver
        assert bloch.solve_mri is feelmri_b200.BlochSimulator.solve_mri
        motion = importlib.import_module("feelmri.Motion")
        assert motion.POD.calculate_pod is calculate_pod_on_device
        bloch.BlochSolver = object  # imported before a second install: patched at once
        feelmri_b200.install_as_feelmri()
        assert bloch.BlochSolver is BlochSolver
    finally:
        sys.path.remove(str(tmp_path))
        for k in [k for k in sys.modules if k == "feelmri" or k.startswith("feelmri.")]:
            del sys.modules[k]
        sys.modules.update(saved)
        feelmri_b200._PATCHES.clear()


def test_gather_data_reduces_host_data_on_cuda_under_nccl():
    # NCCL reduces CUDA tensors only: host (numpy) data must be staged on the
    # current CUDA device; gloo reduces in place on the host
    from feelmri_b200.distributed import reduce_device
    host = torch.zeros(4)
    assert reduce_device("nccl", host, current_cuda=3) == torch.device("cuda", 3)
    assert reduce_device("gloo", host) == torch.device("cpu")
    dev_t = torch.empty(0, device="meta")
    assert reduce_device("nccl", dev_t, current_cuda=0) == torch.device("cuda", 0)


def test_simulate_batch_groups_are_consecutive_and_balanced():
    # simulate_batch stages and launches its requests in groups: every request
    # in exactly one group, in order, and the groups' work close to equal
    from types import SimpleNamespace
    from feelmri_b200.serving import _split_by_work
    rng = np.random.default_rng(3)
    reqs = [SimpleNamespace(work=float(w)) for w in rng.uniform(1.0, 10.0, 64)]
    total = sum(r.work for r in reqs)
    for parts in (1, 2, 4, 7):
        groups = _split_by_work(reqs, parts)
        assert 1 <= len(groups) <= parts
        assert [r for g in groups for r in g] == reqs
        if parts > 1:
            sums = [sum(r.work for r in g) for g in groups]
            assert max(sums) <= total / parts + 10.0
    assert _split_by_work([], 3) == []
