"""ORACLE -- test infrastructure, not product code.

NumPy float64 restatement of the reference's hot path, the accuracy reference
for the GPU forms (relative L2 errors are stated against it).

* bloch():  cpp/feelmri/BlochSimulator.cpp:12-148 / :151-277 in float64.
* signal(): cpp/feelmri/MRI.cpp:38-159 / :196-298 in float64, with
  pi_mode='float' (2 * float32(pi), as MRI.h:13 / MRI.cpp:73 build it) or
  'exact'.  Vectorised over samples in chunks: identical mathematics, node sums
  by numpy's pairwise summation.
* lumped_p1(): exact P1 lumped weights (vol / 4 per element vertex).
* nudft_adjoint(): the exact adjoint NUDFT as a direct sum, the check of the
  GPU reconstruction operators (feelmri_b200.Recon); the reference's own
  reconstruction uses pynufft's gridding approximation (not installed here),
  against which the GPU operators are unpinned.
"""
from __future__ import annotations

import numpy as np

FLOAT_PI = float(np.float32(np.pi))


def bloch(r0, T1, T2, dB, M0, gamma, rf, G, dt, Mxy0, Mz0, disp=None, history=False):
    """Float64 Bloch sweep; disp: (n_t, N, 3) per call (entry i+1 for step i)."""
    r0 = np.asarray(r0, np.float64)
    N = r0.shape[0]
    rf = np.asarray(rf, np.complex128).reshape(-1)
    n_t = rf.shape[0]
    G = np.asarray(G, np.float64).reshape(n_t, 3)
    dt = np.asarray(dt, np.float64).reshape(-1)
    T1 = np.asarray(T1, np.float64).reshape(-1)
    T2 = np.asarray(T2, np.float64).reshape(-1)
    dB = np.asarray(dB, np.float64).reshape(-1)
    m = np.asarray(Mxy0, np.complex128).reshape(-1).copy()
    mz = np.asarray(Mz0, np.float64).reshape(-1).copy()
    hist_m = [m.copy()] if history else None
    hist_z = [mz.copy()] if history else None
    for i in range(n_t - 1):
        d = dt[i + 1]
        e1 = np.exp(-d / T1)
        e2 = np.exp(-d / T2)
        x = r0 if disp is None else r0 + np.asarray(disp[i + 1], np.float64)
        Bz = x @ G[i + 1] + dB
        Bn = np.maximum(np.sqrt(Bz * Bz + abs(rf[i + 1]) ** 2), 1e-12)
        hp = -0.5 * gamma * d * Bn
        c, s = np.cos(hp), np.sin(hp)
        alpha = c - 1j * (Bz / Bn) * s
        beta = -1j * (rf[i + 1] / Bn) * s
        ca = np.conj(alpha)
        mn = 2 * ca * beta * mz + ca * ca * m - beta * beta * np.conj(m)
        mzn = (np.abs(alpha) ** 2 - np.abs(beta) ** 2) * mz - 2 * np.real(alpha * beta * np.conj(m))
        m = mn * e2
        mz = mzn * e1 + (1 - e1) * M0
        if history:
            hist_m.append(m.copy())
            hist_z.append(mz.copy())
    if history:
        return np.stack(hist_m, axis=1), np.stack(hist_z, axis=1)
    return m, mz


def run_starts(t_flat: np.ndarray) -> np.ndarray:
    if t_flat.size == 0:
        return np.zeros(0, np.int64)
    return np.concatenate(([0], np.flatnonzero(t_flat[1:] != t_flat[:-1]) + 1))


def signal(M, kx, ky, kz, t, r0, phi, T2, Mxy, disp=None, pi_mode="exact", sample_idx=None, chunk=256):
    """Float64 k-space (n_ro, n_lines, n_kz, V); with sample_idx, only those
    flat sample indices (returned as (len(sample_idx), V))."""
    two_pi = 2.0 * (np.pi if pi_mode == "exact" else FLOAT_PI)
    grid = np.shape(kx)
    kx = np.asarray(kx, np.float64).reshape(-1)
    ky = np.asarray(ky, np.float64).reshape(-1)
    kz = np.asarray(kz, np.float64).reshape(-1)
    tf = np.asarray(t, np.float64).reshape(-1)
    r0 = np.asarray(r0, np.float64)
    N = r0.shape[0]
    Mxy = np.asarray(Mxy, np.complex128).reshape(N, -1)
    V = Mxy.shape[1]
    MM = np.asarray(M @ Mxy, np.complex128)
    phi = np.asarray(phi, np.float64).reshape(-1)
    invT2 = 1.0 / np.asarray(T2, np.float64).reshape(-1)
    starts = run_starts(np.asarray(t).reshape(-1))
    run_of = np.zeros(tf.size, np.int64)
    if tf.size:
        run_of[starts[1:]] = 1
        run_of = np.cumsum(run_of)
    sel = np.arange(tf.size) if sample_idx is None else np.asarray(sample_idx)
    out = np.zeros((sel.size, V), np.complex128)
    # group the selected samples by run
    order = np.argsort(run_of[sel], kind="stable")
    sel_sorted = sel[order]
    runs = run_of[sel_sorted]
    bounds = np.concatenate(([0], np.flatnonzero(runs[1:] != runs[:-1]) + 1, [sel_sorted.size]))
    for b0, b1 in zip(bounds[:-1], bounds[1:]):
        if b1 <= b0:
            continue
        g = runs[b0]
        ts = tf[starts[g]]
        x = r0 if disp is None else r0 + np.asarray(disp[g], np.float64)
        W = MM * np.exp(-ts * invT2)[:, None]
        ph_off = phi * ts
        idx = sel_sorted[b0:b1]
        for c0 in range(0, idx.size, chunk):
            ii = idx[c0:c0 + chunk]
            k = np.stack([kx[ii], ky[ii], kz[ii]], axis=1) * two_pi
            ph = -(k @ x.T) + ph_off[None, :]
            E = np.exp(1j * ph)
            out[order[b0 + c0:b0 + c0 + ii.size]] = E @ W
    if sample_idx is None:
        return out.reshape(*grid, V)
    return out


def nudft_adjoint(kx, ky, kz, kdata, points, dcw=None, pi_mode="float", chunk=512):
    """Float64 exact adjoint NUDFT I[n, c] = sum_s w_s K[s, c] exp(+i 2 pi k_s . x_n)
    at `points` (n, 3); the direct sum, independent of the Signal restatement.
    The GPU reconstruction (feelmri_b200.Recon) uses the Signal's float pi."""
    two_pi = 2.0 * (np.pi if pi_mode == "exact" else FLOAT_PI)
    k = np.stack([np.asarray(a, np.float64).reshape(-1) for a in (kx, ky, kz)], axis=1)
    K = np.asarray(kdata, np.complex128).reshape(k.shape[0], -1)
    if dcw is not None:
        K = K * np.asarray(dcw, np.float64).reshape(-1, 1)
    x = np.asarray(points, np.float64).reshape(-1, 3)
    out = np.zeros((x.shape[0], K.shape[1]), np.complex128)
    for c0 in range(0, x.shape[0], chunk):
        E = np.exp(1j * two_pi * (x[c0:c0 + chunk] @ k.T))
        out[c0:c0 + chunk] = E @ K
    return out


def lumped_p1(elems, nodes) -> np.ndarray:
    """Exact lumped P1 weights: each tetrahedron gives |vol| / 4 to its vertices."""
    nodes = np.asarray(nodes, np.float64)
    X = nodes[elems]
    vol = np.abs(np.linalg.det(X[:, 1:, :] - X[:, :1, :])) / 6.0
    out = np.zeros(nodes.shape[0])
    for i in range(4):
        np.add.at(out, elems[:, i], vol / 4.0)
    return out


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
