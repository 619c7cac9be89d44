"""ORACLE -- test infrastructure, not product code.

CPU restatements of the reference's hot path used only as the checker in
tests/, in __graft_entry__.smoke() and as the timed CPU baseline in bench.py.
The product package (feelmri_b200) never imports this package.

* refsem (oracle/refsem.c, built by oracle/Makefile): the reference's loop
  order and precision (FP32 Bloch, FP32/FP64 Signal, mass assembly with
  setFromTriplets semantics, scipy row sums, tensordot).
* fp64 (oracle/fp64.py): NumPy float64 restatement with exact or
  float-rounded pi, used as the accuracy reference of the GPU forms.

Parity pinning: no golden vectors exist in the reference's tests and its
native modules cannot be built in this container (Eigen is fetched from the
network at configure time).  The oracle is pinned by analytic known answers
(tests/test_oracle_kat.py) and by vectors generated from the reference's own
python/feelmri/Motion.py (tests/golden/).  Against the reference's native
code itself parity is unpinned.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "build"

_libs: dict[str, C.CDLL] = {}

_p = C.c_void_p
_i64 = C.c_int64


def build() -> None:
    """Compiles the C restatement (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib(flavour: str = "strict") -> C.CDLL:
    """flavour: 'strict' (IEEE order) or 'fast' (reference compiler flags)."""
    if flavour in _libs:
        return _libs[flavour]
    path = BUILD / f"liboracle_{flavour}.so"
    if not path.exists():
        build()
    h = C.CDLL(str(path))
    h.oracle_bloch_f32.argtypes = [_i64, _i64] + [_p] * 4 + [C.c_float, C.c_float] + [_p] * 10
    h.oracle_bloch_f32.restype = None
    for name in ("oracle_signal_f32", "oracle_signal_f64"):
        fn = getattr(h, name)
        fn.argtypes = [_i64, _i64, _i64] + [_p] * 12 + [_i64, C.c_int, C.c_int, _p]
        fn.restype = None
    for name in ("oracle_signal_f32_range", "oracle_signal_f64_range"):
        fn = getattr(h, name)
        fn.argtypes = [_i64, _i64, _i64] + [_p] * 12 + [_i64, C.c_int, _i64, _i64, _p]
        fn.restype = None
    for name in ("oracle_tensordot_f32", "oracle_tensordot_f64"):
        fn = getattr(h, name)
        fn.argtypes = [_p, _p, _i64, _i64, _p]
        fn.restype = None
    for name in ("oracle_mass_f32", "oracle_mass_f64"):
        fn = getattr(h, name)
        fn.argtypes = [_i64, C.c_int, _p, _i64, _p, C.c_int, _p, _p, _p, _p, _p]
        fn.restype = _i64
    for name in ("oracle_csc_rowsum_f32", "oracle_csc_rowsum_f64"):
        fn = getattr(h, name)
        fn.argtypes = [_i64, _p, _p, _p, _p]
        fn.restype = None
    h.oracle_max_threads.restype = C.c_int
    _libs[flavour] = h
    return h


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def bloch_f32(r0, T1, T2, dB, M0, gamma, rf, G, dt, Mxy0, Mz0, disp=None, history=True, flavour="strict"):
    """solve_mri<float> restated.  disp: (n_t, N, 3) float32 displacements per
    call (entry 0 = the call at 0.0) or None.  Returns (Mxy, Mz) as (N, n_t)
    when history else the final (N,) state."""
    r0 = _c(r0, np.float32)
    N = r0.shape[0]
    rf = _c(rf, np.complex64).reshape(-1)
    n_t = rf.shape[0]
    args = [_c(T1, np.float32).reshape(-1), _c(T2, np.float32).reshape(-1), _c(dB, np.float32).reshape(-1)]
    G = _c(G, np.float32).reshape(n_t, 3)
    dt = _c(dt, np.float32).reshape(-1)
    Mxy0 = _c(Mxy0, np.complex64).reshape(-1)
    Mz0 = _c(Mz0, np.float32).reshape(-1)
    d = None if disp is None else _c(disp, np.float32)
    if history:
        mh = np.zeros((n_t, N), np.complex64)
        zh = np.zeros((n_t, N), np.float32)
        lib(flavour).oracle_bloch_f32(N, n_t, _ptr(r0), *map(_ptr, args), float(M0), float(gamma), _ptr(rf),
                                      _ptr(G), _ptr(dt), _ptr(Mxy0), _ptr(Mz0), _ptr(d), _ptr(mh), _ptr(zh), None,
                                      None)
        return mh.T, zh.T
    mo = np.zeros(N, np.complex64)
    zo = np.zeros(N, np.float32)
    lib(flavour).oracle_bloch_f32(N, n_t, _ptr(r0), *map(_ptr, args), float(M0), float(gamma), _ptr(rf), _ptr(G),
                                  _ptr(dt), _ptr(Mxy0), _ptr(Mz0), _ptr(d), None, None, _ptr(mo), _ptr(zo))
    return mo, zo


def signal(M_csc, kx, ky, kz, t, r0, phi, T2, Mxy, disp=None, dtype=np.float32, pi_exact=False, threads=1,
           flavour="strict"):
    """Signal<T> restated.  M_csc: scipy CSC (N, N); disp: (n_runs, N, 3) per
    distinct-time run or None.  Returns (n_ro, n_lines, n_kz, V) complex."""
    T = np.dtype(dtype)
    CT = np.complex64 if T == np.float32 else np.complex128
    grid = np.shape(kx)
    S = int(np.prod(grid))
    r0 = _c(r0, T)
    N = r0.shape[0]
    Mxy = _c(Mxy, CT).reshape(N, -1)
    V = Mxy.shape[1]
    indptr = _c(M_csc.indptr, np.int32)
    indices = _c(M_csc.indices, np.int32)
    data = _c(M_csc.data, T)
    arrs = [_c(a, T).reshape(-1) for a in (kx, ky, kz, t)]
    phi = _c(phi, T).reshape(-1)
    T2 = _c(T2, T).reshape(-1)
    d = None if disp is None else _c(disp, T)
    n_runs = 0 if disp is None else d.shape[0]
    out = np.zeros((S, V), CT)
    fn = lib(flavour).oracle_signal_f32 if T == np.float32 else lib(flavour).oracle_signal_f64
    fn(N, V, S, _ptr(indptr), _ptr(indices), _ptr(data), *map(_ptr, arrs), _ptr(r0), _ptr(phi), _ptr(T2),
       _ptr(Mxy), _ptr(d), n_runs, 1 if pi_exact else 0, int(threads), _ptr(out))
    return out.reshape(*grid, V)


def tensordot(modes, weights):
    modes = np.ascontiguousarray(modes)
    P, Cc, M = modes.shape
    out = np.zeros((P, Cc), modes.dtype)
    fn = lib().oracle_tensordot_f32 if modes.dtype == np.float32 else lib().oracle_tensordot_f64
    fn(_ptr(modes), _ptr(np.ascontiguousarray(weights, modes.dtype)), P * Cc, M, _ptr(out))
    return out


def mass_csc(elems, nodes, qweights, tab):
    """(indptr, indices, data) as MassAssemble<T> + setFromTriplets produce them."""
    nodes = np.ascontiguousarray(nodes)
    T = nodes.dtype
    elems = _c(elems, np.int32)
    E, nb = elems.shape
    N = nodes.shape[0]
    qw = _c(qweights, T)
    tab = _c(tab, T)
    fn = lib().oracle_mass_f32 if T == np.float32 else lib().oracle_mass_f64
    nnz = fn(E, nb, _ptr(elems), N, _ptr(nodes), qw.shape[0], _ptr(qw), _ptr(tab), None, None, None)
    indptr = np.zeros(N + 1, np.int32)
    indices = np.zeros(nnz, np.int32)
    data = np.zeros(nnz, T)
    fn(E, nb, _ptr(elems), N, _ptr(nodes), qw.shape[0], _ptr(qw), _ptr(tab), _ptr(indptr), _ptr(indices),
       _ptr(data))
    return indptr, indices, data


def csc_rowsum(indptr, indices, data):
    N = indptr.shape[0] - 1
    y = np.zeros(N, data.dtype)
    fn = lib().oracle_csc_rowsum_f32 if data.dtype == np.float32 else lib().oracle_csc_rowsum_f64
    fn(N, _ptr(_c(indptr, np.int32)), _ptr(_c(indices, np.int32)), _ptr(np.ascontiguousarray(data)), _ptr(y))
    return y


def max_threads() -> int:
    return int(lib("fast").oracle_max_threads())
