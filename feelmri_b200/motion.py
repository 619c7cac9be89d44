"""Motion on the device: spline-driven displacement fields and the device
POD construction.

Two things live here.

1. ``SplineMotion`` -- a displacement field u(t) = sum_k u_k(t), each term
   either a mode expansion Phi_k a_k(t) (a_k a piecewise polynomial, optionally
   scaled by t to turn a velocity basis into a displacement) or a rigid shift
   d_k s_k(t) along a fixed direction.  It is the library's own way to state a
   motion from explicit modes and spline coefficients (synthetic phantoms,
   motion fitted elsewhere).  It lowers to the same device descriptor as the
   reference's Motion.py callables (``fm_motion_terms`` below), so the Bloch
   and Signal kernels evaluate it on the GPU, and its host ``__call__``
   evaluates the same arithmetic in numpy for checks.

2. ``snapshot_pod`` / ``calculate_pod_on_device`` -- the method-of-snapshots
   POD of a (P, C, t) history with the two large products on the GPU (the
   t x t Gram matrix and the projections, FP64 sums in a fixed order; see
   csrc/pod_build.cu) and the small t x t symmetric eigenproblem on the host.
   ``calculate_pod_on_device`` has the contract of the reference's
   ``POD.calculate_pod`` (python/feelmri/Motion.py:174-217): it reads
   ``times``, ``data``, ``n_modes`` and ``local_to_global_map`` from any
   POD-like object and returns ``(modes (P, C, r), weights (t, r))``;
   ``feelmri_b200.install_as_feelmri(device_pod=True)`` installs it in place
   of the reference's method, so unchanged scripts build their POD on the GPU.

Time arithmetic of ``SplineMotion`` (so that the device reproduces it bit for
bit): the evaluation time is the float64 sum t + timeshift, folded into
[0, period) as tau - period * floor(tau / period) in float64 when a period is
set; each polynomial is evaluated in float64 and rounded to float32; a
velocity term multiplies its float32 coefficients by float32(t) (the
unshifted, unfolded time); the float32 mode contraction and the float32 sum
of the terms follow.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["SplineTerm", "SplineMotion", "snapshot_pod", "calculate_pod_on_device"]


@dataclass
class SplineTerm:
    """One term of a SplineMotion.

    kind: "modes" (Phi a(t)), "velocity_modes" (Phi a(t) t) or "rigid"
    (direction s(t)).  coeffs (k, n_intervals, r) float64 and knots
    (n_intervals + 1,) float64 define the piecewise polynomials in the local
    power basis, highest power first (r = 1 for a rigid term).  modes is
    (N, 3, r) float32 for the mode kinds; direction is (3,) float32 for a
    rigid term.  Outside [knots[0], knots[-1]] the term is NaN unless
    extrapolate is set; period folds the time first."""
    kind: str
    coeffs: np.ndarray
    knots: np.ndarray
    modes: np.ndarray | None = None
    direction: np.ndarray | None = None
    period: float | None = None
    extrapolate: bool = False

    def __post_init__(self):
        if self.kind not in ("modes", "velocity_modes", "rigid"):
            raise ValueError(f"unknown term kind {self.kind!r}")
        self.coeffs = np.ascontiguousarray(self.coeffs, np.float64)
        self.knots = np.ascontiguousarray(self.knots, np.float64)
        if self.coeffs.ndim != 3 or self.coeffs.shape[1] != self.knots.shape[0] - 1:
            raise ValueError("coeffs must be (k, len(knots) - 1, r)")
        if self.kind == "rigid":
            if self.coeffs.shape[2] != 1:
                raise ValueError("a rigid term has one polynomial (r = 1)")
            d = np.asarray(self.direction, np.float32).reshape(3)
            self.direction = d
        else:
            m = np.ascontiguousarray(self.modes, np.float32)
            if m.ndim != 3 or m.shape[1] != 3 or m.shape[2] != self.coeffs.shape[2]:
                raise ValueError("modes must be (N, 3, r) with r polynomials")
            self.modes = m
        if self.period is not None:
            self.period = float(self.period)

    def coefficients_at(self, tau: float) -> np.ndarray:
        """float32 values of the r polynomials at the (already shifted and
        folded) time tau: float64 evaluation, then rounding."""
        x = self.knots
        lo, hi = x[0], x[-1]
        if not self.extrapolate and not (lo <= tau <= hi):
            return np.full(self.coeffs.shape[2], np.nan, np.float32)
        # interval i with x[i] <= tau < x[i+1]; the last interval is closed
        i = int(np.searchsorted(x, tau, side="right")) - 1
        i = min(max(i, 0), x.shape[0] - 2)
        h = tau - x[i]
        acc = np.zeros(self.coeffs.shape[2], np.float64)
        powh = 1.0
        k = self.coeffs.shape[0]
        for j in range(k - 1, -1, -1):  # lowest power first
            acc += self.coeffs[j, i] * powh
            powh *= h
        return acc.astype(np.float32)


class SplineMotion:
    """u(t) = sum of SplineTerm contributions, all sharing one timeshift.

    ``update_timeshift`` moves the time origin (BlochSolver sets it to each
    block's start); ``__add__`` concatenates the terms of two motions."""

    def __init__(self, terms, timeshift: float = 0.0):
        self.terms = list(terms)
        if not self.terms:
            raise ValueError("a SplineMotion needs at least one term")
        self.timeshift = float(timeshift)

    @classmethod
    def from_samples(cls, modes, times, samples, *, periodic: bool = True, velocity: bool = False,
                     timeshift: float = 0.0) -> "SplineMotion":
        """Modes (N, 3, r) with coefficient samples (len(times), r) fitted by
        monotone cubic (PCHIP) splines; periodic folds time into
        [0, times[-1])."""
        from scipy.interpolate import PchipInterpolator
        times = np.asarray(times, np.float64)
        samples = np.asarray(samples, np.float64).reshape(times.shape[0], -1)
        fit = PchipInterpolator(times, samples, axis=0)
        term = SplineTerm("velocity_modes" if velocity else "modes", np.asarray(fit.c), np.asarray(fit.x),
                          modes=modes, period=float(times[-1]) if periodic else None)
        return cls([term], timeshift)

    @classmethod
    def rigid(cls, direction, times, samples, *, periodic: bool = False, timeshift: float = 0.0) -> "SplineMotion":
        """A rigid shift along `direction` (normalised) by the PCHIP fit of
        samples(times)."""
        from scipy.interpolate import PchipInterpolator
        times = np.asarray(times, np.float64)
        fit = PchipInterpolator(times, np.asarray(samples, np.float64).reshape(-1, 1), axis=0)
        d = np.asarray(direction, np.float64).reshape(3)
        term = SplineTerm("rigid", np.asarray(fit.c), np.asarray(fit.x), direction=(d / np.linalg.norm(d)),
                          period=float(times[-1]) if periodic else None, extrapolate=True)
        return cls([term], timeshift)

    @property
    def n_nodes(self) -> int | None:
        for t in self.terms:
            if t.modes is not None:
                return t.modes.shape[0]
        return None

    def update_timeshift(self, timeshift) -> None:
        self.timeshift = float(timeshift)

    def __add__(self, other: "SplineMotion") -> "SplineMotion":
        if not isinstance(other, SplineMotion):
            return NotImplemented
        return SplineMotion(self.terms + other.terms, self.timeshift)

    def _tau(self, t: float, term: SplineTerm) -> float:
        tau = float(t) + self.timeshift
        if term.period is not None:
            P = term.period
            tau = tau - P * float(np.floor(tau / P))
        return tau

    def __call__(self, t) -> np.ndarray:
        """(N, 3) float32 displacement at time t (a (1, 3) row when every
        term is rigid)."""
        out = None
        for term in self.terms:
            a = term.coefficients_at(self._tau(t, term))
            if term.kind == "velocity_modes":
                a = (a * np.float32(t)).astype(np.float32)
            if term.kind == "rigid":
                u = (a[0] * term.direction).reshape(1, 3).astype(np.float32)
            else:
                u = np.einsum("ncr,r->nc", term.modes, a).astype(np.float32)
            out = u if out is None else (out + u).astype(np.float32)
        return out

    def fm_motion_terms(self) -> list[dict]:
        """The terms in the form the device lowering reads."""
        return [dict(kind=t.kind, coeffs=t.coeffs, knots=t.knots, modes=t.modes, direction=t.direction,
                     period=t.period, extrapolate=t.extrapolate, timeshift=self.timeshift) for t in self.terms]


# ------------------------------------------------------- POD construction --

def snapshot_pod(times, data, n_modes: int, *, remove_mean: bool = False):
    """Method-of-snapshots POD of data (P, C, t) on the current CUDA device.

    With X the (P*C, t) snapshot matrix: G = X^T X is formed on the GPU (FP64
    sums), its eigenpairs (lambda_j, e_j) are found on the host, the r = n_modes
    largest are kept, and the modes phi_j = X e_j / sqrt(lambda_j) and the
    coefficients a = X^T phi (t, r) are formed on the GPU.  Returns
    (modes (P, C, r), weights (t, r)) in data's floating type."""
    import torch
    from . import ops
    data = np.asarray(data)
    n_t = int(np.asarray(times).shape[0])
    if data.dtype not in (np.float32, np.float64):
        raise TypeError(f"snapshot_pod takes float32 or float64 data, got {data.dtype}")
    if data.size % n_t:
        raise ValueError(f"data of shape {data.shape} does not hold {n_t} snapshots")
    if not 1 <= n_modes <= n_t:
        raise ValueError(f"n_modes must be in [1, {n_t}]")
    X = np.ascontiguousarray(data.reshape(-1, n_t))
    if remove_mean:
        X = X - X.mean(axis=1, keepdims=True, dtype=X.dtype)
    dev = ops.require_cuda()
    Xd = torch.from_numpy(X).to(dev)
    gram = ops.pod_gram(Xd).cpu().numpy()
    lam, vec = np.linalg.eigh(gram.astype(X.dtype))
    keep = np.argsort(lam)[::-1][:n_modes]
    scale = vec[:, keep] / np.sqrt(lam[keep])[None, :]
    phi, coef = ops.pod_project(Xd, torch.from_numpy(np.ascontiguousarray(scale, np.float64)).to(dev))
    modes = phi.cpu().numpy().reshape(data.shape[0], -1, n_modes)
    return modes, coef.cpu().numpy().astype(X.dtype)


def calculate_pod_on_device(pod, remove_mean: bool = False):
    """Drop-in body for a POD-like object's ``calculate_pod`` (the contract of
    python/feelmri/Motion.py:174-217): reads pod.times, pod.data, pod.n_modes
    and pod.local_to_global_map, returns (modes, weights) with the modes
    restricted to the local nodes when a map is set."""
    modes, weights = snapshot_pod(pod.times, pod.data, int(pod.n_modes), remove_mean=remove_mean)
    l2g = getattr(pod, "local_to_global_map", None)
    if l2g is not None:
        modes = modes[l2g, :, :]
    return modes, weights
