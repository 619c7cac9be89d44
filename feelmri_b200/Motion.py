"""Motion callables with the interface of python/feelmri/Motion.py.

POD, PODVelocity, PODSum and RespiratoryMotion hold the same state under the
same attribute names as the reference's classes (_modes, _pp_batch,
timeshift, _period, _weights, interpolator, direction, pod1/pod2) so that the
GPU entry points lower either set of classes to device motion descriptors
(feelmri_b200._motion).  Construction is host work done once, as in the
reference: snapshot POD through an eigen-decomposition of the (t x t)
covariance (Motion.py:174-217) and a per-mode spline of the weights
(Motion.py:219-235) gathered into one batched PPoly (Motion.py:128-137).

Calling one of these objects evaluates it the reference's way: the spline in
float64 on the host, cast to float32 (Motion.py:237-238), then the modes x
weights product through feelmri_b200.POD.tensordot_modes_weights (GPU).
"""
from __future__ import annotations

from collections.abc import Callable

import numpy as np
from scipy.interpolate import Akima1DInterpolator, CubicSpline, PchipInterpolator, PPoly

__all__ = ["POD", "PODVelocity", "PODSum", "RespiratoryMotion"]

_SPLINES = {"AkimaSpline": Akima1DInterpolator, "CubicSpline": CubicSpline, "Pchip": PchipInterpolator}


def _periodic_fold(period):
    if period is None:
        return lambda x: x

    def _fold(x, T=period):
        # x - T floor(x / T), in the NumPy types of x and T (Motion.py:146-148)
        return x - T * np.floor(x / T)
    return _fold


class RespiratoryMotion:
    """Rigid displacement along a direction from a 1-D spline (Motion.py:15-109)."""

    def __init__(self, times, data, timeshift=0.0, is_periodic=False, remove_mean=False,
                 direction=np.array([1, 0, 0], dtype=np.float32), interpolation_method="Pchip"):
        self.times = np.asarray(times).astype(np.float32)
        self.data = np.asarray(data).astype(np.float32)
        self.timeshift = timeshift
        self.is_periodic = is_periodic
        self.remove_mean = remove_mean
        d = np.asarray(direction)
        self.direction = (d.reshape((1, 3)) / np.linalg.norm(d)).astype(np.float32)
        self.interpolation_method = interpolation_method
        self.interpolator = self.calculate_interpolator()
        self._period = self.times[-1] if self.is_periodic else None
        self._fold_time = _periodic_fold(self._period)

    def __add__(self, other):
        return PODSum(self, other)

    def __call__(self, t):
        return self._evaluate_motion(t) * self.direction

    def calculate_interpolator(self):
        data = self.data
        if self.remove_mean:
            data -= np.mean(self.data, axis=0, dtype=np.float32)
        if self.interpolation_method not in _SPLINES:
            raise ValueError(f"Interpolation method '{self.interpolation_method}' not recognized.")
        if self.interpolation_method == "CubicSpline":
            return CubicSpline(self.times, data, bc_type="natural")
        return _SPLINES[self.interpolation_method](self.times, data)

    def _evaluate_motion(self, t):
        t = self._fold_time(t + self.timeshift)
        return self.interpolator(t).astype(np.float32)

    def update_timeshift(self, timeshift):
        self.timeshift = timeshift


class POD:
    """Snapshot POD of nodal vectors (P, C, t) with spline-interpolated weights."""

    def __init__(self, times, data, global_to_local=None, n_modes=5, is_periodic=False,
                 interpolation_method="Pchip", timeshift=0.0, *, backend="numpy"):
        """backend="cuda" forms the snapshot products (X^T X, X E, X^T phi)
        on the GPU (fm_pod_gram_*, fm_pod_project_*) with FP64 sums; the
        t x t eigenproblem and the spline fit stay on the host as in the
        reference.  The default "numpy" is the reference's computation."""
        if backend not in ("numpy", "cuda"):
            raise ValueError(f"backend must be 'numpy' or 'cuda'; got {backend!r}")
        self.backend = backend
        self.times = times
        self.data = data
        self.local_to_global_map = global_to_local
        self.n_modes = n_modes
        self.timeshift = timeshift
        self.is_periodic = is_periodic
        self.interpolation_method = interpolation_method
        self.modes, self.weights = self.calculate_pod(remove_mean=False)
        self.spline_coeffs = self.spline_fit()
        x0 = self.spline_coeffs[0].x
        for s in self.spline_coeffs:
            if not isinstance(s, PPoly):
                raise TypeError("Use CubicSpline/Pchip/Akima (PPoly subclasses)")
            if not np.array_equal(s.x, x0):
                raise ValueError("knots differ between modes")
        C = np.stack([s.c for s in self.spline_coeffs], axis=-1)
        self._pp_batch = PPoly(C, x0, extrapolate=False)
        self._modes = np.asarray(self.modes, dtype=np.float32, order="C")
        self._period = self.times[-1] if self.is_periodic else None
        self._weights = np.zeros([self.n_modes], dtype=np.float32, order="C")
        self._fold_time = _periodic_fold(self._period)

    def __repr__(self):
        return (f"POD(n_modes={self.n_modes}, interpolation_method='{self.interpolation_method}', "
                f"is_periodic={self.is_periodic})")

    def __add__(self, other):
        return PODSum(self, other)

    def __call__(self, t):
        return self._evaluate_trajectory(t)

    def calculate_pod(self, remove_mean=False):
        n_t = self.times.shape[0]
        flat = self.data.reshape(-1, n_t)
        if remove_mean:
            flat = flat - np.mean(flat, axis=1, keepdims=True)
        device = self.backend == "cuda" and flat.dtype in (np.float32, np.float64)
        if device:
            import torch
            from . import ops
            X = torch.from_numpy(np.ascontiguousarray(flat)).to(ops.require_cuda())
            cov = ops.pod_gram(X).cpu().numpy().astype(flat.dtype)
        else:
            cov = flat.T @ flat
        vals, vecs = np.linalg.eigh(cov)
        order = np.argsort(vals)[::-1][: self.n_modes]
        vals, vecs = vals[order], vecs[:, order]
        E = vecs / np.sqrt(vals).reshape(1, -1)
        if device:
            phi_d, w_d = ops.pod_project(X, torch.from_numpy(np.ascontiguousarray(E, np.float64)).to(X.device))
            phi, weights = phi_d.cpu().numpy(), w_d.cpu().numpy().astype(flat.dtype)
        else:
            phi = flat @ E
            weights = np.einsum("pn, pt -> nt", flat, phi)
        phi = phi.reshape((self.data.shape[0], -1, self.n_modes))
        if self.local_to_global_map is not None:
            phi = phi[self.local_to_global_map, :, :]
        return phi, weights

    def spline_fit(self):
        if self.interpolation_method not in _SPLINES:
            raise ValueError(f"Interpolation method '{self.interpolation_method}' not recognized.")
        interp = _SPLINES[self.interpolation_method]
        return [interp(self.times, self.weights[:, i]) for i in range(self.n_modes)]

    def _evaluate_weights(self, t):
        self._weights[:] = self._pp_batch(t).astype(self._weights.dtype, copy=False)

    def _evaluate_trajectory(self, t):
        from .POD import tensordot_modes_weights
        self._evaluate_weights(self._fold_time(t + self.timeshift))
        return tensordot_modes_weights(self._modes, self._weights)

    def update_timeshift(self, timeshift):
        self.timeshift = timeshift


class PODVelocity(POD):
    """POD of velocities: the weights are scaled by the unfolded time (Motion.py:272-290)."""

    def _evaluate_trajectory(self, t):
        from .POD import tensordot_modes_weights
        self._evaluate_weights(self._fold_time(t + self.timeshift))
        self._weights *= t
        return tensordot_modes_weights(self._modes, self._weights)


class PODSum:
    """Sum of two motion callables (Motion.py:293-317)."""

    def __init__(self, pod1, pod2: Callable):
        self.pod1 = pod1
        self.pod2 = pod2
        self.timeshift = 0.0

    def __call__(self, t):
        return self.pod1(t) + self.pod2(t)

    def update_timeshift(self, timeshift):
        self.pod1.update_timeshift(timeshift)
        self.pod2.update_timeshift(timeshift)
        self.timeshift = timeshift

    def __add__(self, other):
        return PODSum(self, other)
