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
    a = bench.build_batch_case(n_phantoms=6)
    b = bench.build_batch_case(n_phantoms=6)
    assert [c["N"] for c in a] == [c["N"] for c in b]
    for c in a:
        assert 4_000 <= c["N"] <= 320_000
        assert 1 <= c["coils"].shape[1] <= 2
        assert c["traj"].shape[2] >= 8  # every trajectory is a kz stack (factorable slabs)


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
    from feelmri_b200.Motion import PODSum
    N = 50
    a = W.sinusoidal_pod(N, n_modes=2, n_frames=5)
    b = W.sinusoidal_pod(N, n_modes=1, n_frames=5, seed=3)
    c = W.sinusoidal_pod(N, n_modes=3, n_frames=6, seed=4)
    for obj in (a, PODSum(a, b), PODSum(PODSum(a, b), c)):
        for t0 in (0.0, np.float32(2.5), np.float64(7.25), 3):
            obj.update_timeshift(t0)
            low = lower(obj, N, torch.device("cpu"))
            got = term_timeshifts(obj)
            want = [(low.struct.terms[k].timeshift, low.struct.terms[k].timeshift_kind)
                    for k in range(low.struct.n_terms)]
            assert got == want


def test_recon_grid_and_analytic_weights():
    # voxel centres on the DFT-centred grid; the analytic density weights of
    # Recon.py:108-146 restated (ramp for radials, readout speed for spirals)
    from feelmri_b200 import Recon
    X, Y, Z = Recon.grid_points((4, 5, 1), (0.08, 0.1, 0.01))
    np.testing.assert_allclose(X[:, 0, 0], np.array([-2, -1, 0, 1]) * 0.02, atol=1e-7)
    np.testing.assert_allclose(Y[0, :, 0], np.array([-2, -1, 0, 1, 2]) * 0.02, atol=1e-7)
    assert np.all(Z == 0)
    R, L, S = 6, 4, 2
    rng = np.random.default_rng(0)
    kx, ky, kz = (rng.normal(size=(R, L, S)) for _ in range(3))
    w = Recon.dcf_radial_stack(kx, ky)
    r = np.sqrt(kx ** 2 + ky ** 2)
    np.testing.assert_allclose(w, (r / (r.mean(axis=(0, 1), keepdims=True) + 1e-6)).ravel(), rtol=1e-6)
    ws = Recon.dcf_local_speed_readout(kx, ky, kz).reshape(R, L, S)
    dk = np.sqrt(np.diff(kx, axis=0) ** 2 + np.diff(ky, axis=0) ** 2 + np.diff(kz, axis=0) ** 2)
    mid = 0.5 * (dk[:-1] + dk[1:])
    full = np.concatenate([dk[:1], mid, dk[-1:]], axis=0)
    np.testing.assert_allclose(ws, full / (full.mean(axis=0, keepdims=True) + 1e-8), rtol=1e-5)
