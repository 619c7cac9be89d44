"""Argument conversion with the rules of the reference's pybind11 bindings.

pybind11 resolves an overloaded function in two passes: first every overload
is tried without implicit conversion, then every overload again with
conversion, in registration order.  The casters involved behave as follows
(pybind11 eigen/matrix.h, eigen/tensor.h, cast.h):

* dense Eigen matrix / array, no-convert pass: the argument must already be a
  numpy array of exactly the scalar dtype; convert pass: anything numpy can
  turn into an array, force-cast to the scalar dtype;
* Eigen tensor: the same, plus the exact number of dimensions;
* Eigen sparse: conversion is unconditional, through
  scipy.sparse.csc_matrix(obj) with the data force-cast to the scalar type;
* float: a Python float (numpy.float64 is one) without conversion, anything
  with __float__ with it; int: never a float;
* std::vector<T>: any sequence that is not str/bytes, item by item;
* py::function: any callable; py::none: only None.

A failed match raises TypeError, as pybind11 does.
"""
from __future__ import annotations

import numpy as np


class NoMatch(Exception):
    """The argument does not fit the caster in this pass."""


def dense(obj, dtype, convert: bool, rows=None, cols=None, vector: bool = False) -> np.ndarray:
    """Eigen Matrix/Array caster.  rows/cols are fixed extents (None = Dynamic);
    vector=True for compile-time column vectors (Matrix<T, Dynamic, 1>)."""
    dtype = np.dtype(dtype)
    if not convert:
        if not isinstance(obj, np.ndarray) or obj.dtype != dtype:
            raise NoMatch
        arr = obj
    else:
        try:
            arr = np.asarray(obj)
        except Exception as exc:  # noqa: BLE001 - any failure means "no match"
            raise NoMatch from exc
        if arr.dtype == object:
            raise NoMatch
    if arr.ndim == 2:
        r, c = arr.shape
        if (rows is not None and r != rows) or (cols is not None and c != cols):
            raise NoMatch
    elif arr.ndim == 1:
        n = arr.shape[0]
        if vector:
            pass
        elif rows is not None and cols is not None:
            raise NoMatch  # fixed-size non-vector types take no 1-D input
        elif cols is not None:
            if cols != n:
                raise NoMatch
            arr = arr.reshape(1, n)  # one row of the fixed width
        else:
            if rows is not None and rows != n:
                raise NoMatch
            arr = arr.reshape(n, 1)  # dynamic: a column
    else:
        raise NoMatch
    if vector and arr.ndim == 2:
        if arr.shape[1] != 1:
            raise NoMatch
        arr = arr[:, 0]
    if arr.dtype != dtype:
        with np.errstate(all="ignore"):
            arr = _force_cast(arr, dtype)
    return arr


def _force_cast(arr: np.ndarray, dtype: np.dtype) -> np.ndarray:
    if np.iscomplexobj(arr) and dtype.kind != "c":
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            return arr.real.astype(dtype)
    return arr.astype(dtype)


def tensor(obj, dtype, ndim: int, convert: bool) -> np.ndarray:
    """Eigen Tensor<T, ndim> caster."""
    dtype = np.dtype(dtype)
    if not convert:
        if not isinstance(obj, np.ndarray) or obj.dtype != dtype:
            raise NoMatch
        arr = obj
    else:
        try:
            arr = np.asarray(obj)
        except Exception as exc:  # noqa: BLE001
            raise NoMatch from exc
        if arr.dtype == object:
            raise NoMatch
        if arr.dtype != dtype:
            with np.errstate(all="ignore"):
                arr = _force_cast(arr, dtype)
    if arr.ndim != ndim:
        raise NoMatch
    return arr


def sequence_of(obj, fn):
    if isinstance(obj, (str, bytes)) or not hasattr(obj, "__len__") or not hasattr(obj, "__getitem__"):
        raise NoMatch
    return [fn(x) for x in obj]


def sparse_csc(obj, dtype):
    """Eigen SparseMatrix<T> (column-major) caster.

    A float lil_matrix (the lumped mass of the reference's examples) is
    converted by the native _hostconv.lil_to_csc, which yields the arrays of
    scipy.sparse.csc_matrix(obj); every other input, and any lil that the
    native pass declines, goes through scipy."""
    import scipy.sparse as sp
    if isinstance(obj, sp.lil_matrix) and obj.dtype in (np.float64, np.float32):
        fast = _lil_to_csc(obj)
        if fast is not None:
            indptr, indices, data = fast
            if data.dtype != np.dtype(dtype):
                data = _force_cast(data.astype(obj.dtype, copy=False), np.dtype(dtype))
            return obj.shape, indptr, indices, data
    try:
        if type(obj) is not sp.csc_matrix:
            obj = sp.csc_matrix(obj)
    except Exception as exc:  # noqa: BLE001
        raise NoMatch from exc
    data = np.asarray(obj.data)
    if data.dtype != np.dtype(dtype):
        data = _force_cast(data, np.dtype(dtype))
    indices = np.asarray(obj.indices).astype(np.int32, copy=False)
    indptr = np.asarray(obj.indptr).astype(np.int32, copy=False)
    return obj.shape, indptr, indices, data


def _lil_to_csc(m):
    try:
        from . import _hostconv
    except ImportError as exc:
        raise ImportError("feelmri_b200._hostconv is not built; run `python -m feelmri_b200.build`") from exc
    n_rows, n_cols = m.shape
    return _hostconv.lil_to_csc(m.rows, m.data, n_rows, n_cols)


def py_float(obj, convert: bool) -> float:
    if not convert:
        if not isinstance(obj, float):
            raise NoMatch
        return float(obj)
    try:
        return float(obj)
    except Exception as exc:  # noqa: BLE001
        raise NoMatch from exc


def py_int(obj, convert: bool) -> int:
    if isinstance(obj, (float, np.floating)):
        raise NoMatch
    if isinstance(obj, (int, np.integer)):
        return int(obj)
    if hasattr(obj, "__index__"):
        return int(obj.__index__())
    if convert:
        try:
            return int(obj)
        except Exception as exc:  # noqa: BLE001
            raise NoMatch from exc
    raise NoMatch


def function_or_none(obj, want_none: bool):
    if want_none:
        if obj is not None:
            raise NoMatch
        return None
    if obj is None or not callable(obj):
        raise NoMatch
    return obj


def no_overload(name: str, args) -> TypeError:
    kinds = ", ".join(type(a).__name__ for a in args)
    return TypeError(f"{name}(): incompatible function arguments; invoked with types ({kinds})")
