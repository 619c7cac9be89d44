"""Test doubles of the reference's motion callables (python/feelmri/Motion.py).

The device lowering (feelmri_b200._motion) recognises the reference's
classes by name and reads their state: `_modes`, `_pp_batch`, `timeshift`,
`_period`, `_weights` for POD / PODVelocity (Motion.py:110-290),
`interpolator`, `direction` for RespiratoryMotion (Motion.py:15-109) and
`pod1` / `pod2` for PODSum (Motion.py:293-317).  The doubles below carry that
state, built directly from given modes and spline data instead of from
snapshots, so that tests can hand the lowering objects shaped like the
reference's without the reference being importable (on the GPU machine it is
not).  Their evaluation is the motion model itself, written for checking:
shift, periodic fold in the NumPy types of t and the period, float64 spline
evaluation rounded to float32, the velocity scaling by the unshifted time,
and a float32 mode contraction.  They are test infrastructure only.
"""
from __future__ import annotations

import numpy as np
from scipy.interpolate import PchipInterpolator, PPoly


def _folder(period):
    if period is None:
        return lambda x: x
    return lambda x: x - period * np.floor(x / period)


class POD:
    """State of a reference POD: modes (N, 3, r) and a batched PPoly."""

    def __call__(self, t):
        return self._evaluate_trajectory(t)

    def _evaluate_weights(self, t):
        self._weights[:] = self._pp_batch(t).astype(self._weights.dtype, copy=False)

    def _evaluate_trajectory(self, t):
        self._evaluate_weights(self._fold_time(t + self.timeshift))
        return np.einsum("ncr,r->nc", self._modes, self._weights).astype(np.float32)

    def update_timeshift(self, timeshift):
        self.timeshift = timeshift

    def __add__(self, other):
        return PODSum(self, other)


class PODVelocity(POD):
    """A POD whose weights are scaled by the unshifted call time."""

    def _evaluate_trajectory(self, t):
        self._evaluate_weights(self._fold_time(t + self.timeshift))
        self._weights *= t
        return np.einsum("ncr,r->nc", self._modes, self._weights).astype(np.float32)


class RespiratoryMotion:
    """State of a reference RespiratoryMotion: a scalar spline and a direction."""

    def __call__(self, t):
        return self._evaluate_motion(t) * self.direction

    def _evaluate_motion(self, t):
        return self.interpolator(self._fold_time(t + self.timeshift)).astype(np.float32)

    def update_timeshift(self, timeshift):
        self.timeshift = timeshift

    def __add__(self, other):
        return PODSum(self, other)


class PODSum:
    def __init__(self, pod1, pod2):
        self.pod1, self.pod2 = pod1, pod2
        self.timeshift = 0.0

    def __call__(self, t):
        return self.pod1(t) + self.pod2(t)

    def update_timeshift(self, timeshift):
        self.pod1.update_timeshift(timeshift)
        self.pod2.update_timeshift(timeshift)
        self.timeshift = timeshift

    def __add__(self, other):
        return PODSum(self, other)


def pod_from_ppoly(c, x, modes, *, velocity=False, extrapolate=False, timeshift=0.0, period=None):
    obj = (PODVelocity if velocity else POD).__new__(PODVelocity if velocity else POD)
    obj._pp_batch = PPoly(np.asarray(c), np.asarray(x), extrapolate=extrapolate)
    obj._modes = np.ascontiguousarray(modes, np.float32)
    obj.n_modes = obj._modes.shape[2]
    obj._weights = np.zeros(obj.n_modes, np.float32)
    obj.timeshift = timeshift
    obj._period = period
    obj._fold_time = _folder(period)
    return obj


def pod_from_samples(modes, times, samples, *, velocity=False, periodic=True, timeshift=0.0):
    """Modes with PCHIP-fitted weight samples (len(times), r); the period is
    times[-1] in the type of `times`, as the reference takes it."""
    times = np.asarray(times)
    fit = PchipInterpolator(times, np.asarray(samples, np.float64), axis=0)
    return pod_from_ppoly(fit.c, fit.x, modes, velocity=velocity, timeshift=timeshift,
                          period=times[-1] if periodic else None)


def respiratory_from_ppoly(c, x, direction, *, extrapolate=True, timeshift=0.0, period=None):
    obj = RespiratoryMotion.__new__(RespiratoryMotion)
    obj.interpolator = PPoly(np.asarray(c), np.asarray(x), extrapolate=extrapolate)
    obj.direction = np.asarray(direction, np.float32).reshape(1, 3)
    obj.timeshift = timeshift
    obj._period = period
    obj._fold_time = _folder(period)
    return obj
