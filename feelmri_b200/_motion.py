"""Lowering of motion callables to the device motion descriptor.

The reference's native routines call a Python `pod_trajectory(t)` once per
Bloch step (cpp/feelmri/BlochSimulator.cpp:44, :86) and once per distinct
readout time (cpp/feelmri/MRI.cpp:50, :114).  For the callables of
python/feelmri/Motion.py the arithmetic of that call is reproduced on the GPU
(see csrc/motion.cuh): this module reads their state (PPoly coefficients and
breakpoints, POD modes, timeshift, period, direction) into an fm_motion
struct.  Objects that state their device form themselves through
fm_motion_terms() (feelmri_b200.motion.SplineMotion) are lowered from that
statement.  Any other callable is sampled at exactly the times the reference
would call it, and its outputs are uploaded as a displacement table.
"""
from __future__ import annotations

import weakref
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L

_POD_NAMES = {"POD": L.FM_TERM_POD, "PODVelocity": L.FM_TERM_POD_VELOCITY}


def num_kind(v) -> int | None:
    """NumPy-2 promotion class of a scalar: weak Python float, float32 or float64."""
    if v is None:
        return L.FM_NUM_NONE
    if isinstance(v, np.ndarray):
        if v.ndim != 0:
            return None
        v = v[()]
    if isinstance(v, np.float32):
        return L.FM_NUM_F32
    if isinstance(v, (np.float64, np.integer)):
        return L.FM_NUM_F64
    if isinstance(v, np.bool_):
        return L.FM_NUM_F64
    if isinstance(v, np.generic):
        return None  # float16, longdouble, complex: not lowered
    if isinstance(v, (float, int)):
        return L.FM_NUM_PYFLOAT
    return None


def _defined_by(obj, attr: str, owner_names) -> bool:
    """True when obj.<attr> comes from a class named in owner_names (so a user
    subclass that overrides the evaluation is not lowered)."""
    for klass in type(obj).__mro__:
        if attr in klass.__dict__:
            return klass.__name__ in owner_names
    return False


class _DeviceCache:
    """Device copies of host arrays, keyed by the identity of the ndarray and
    invalidated when the array object dies or its buffer/shape changes."""

    def __init__(self):
        self._store: dict[tuple, tuple] = {}

    def get(self, arr: np.ndarray, dtype: torch.dtype, device: torch.device) -> torch.Tensor:
        key = (id(arr), str(device), dtype)
        ent = self._store.get(key)
        sig = (arr.__array_interface__["data"][0], arr.shape, arr.dtype.str)
        if ent is not None:
            ref, esig, tensor = ent
            if ref() is arr and esig == sig:
                return tensor
        src = np.ascontiguousarray(arr)
        tensor = torch.from_numpy(src).to(device=device, dtype=dtype)
        try:
            ref = weakref.ref(arr)
        except TypeError:
            return tensor
        self._store[key] = (ref, sig, tensor)
        if len(self._store) > 64:
            for k in [k for k, (r, _, _) in self._store.items() if r() is None]:
                del self._store[k]
        return tensor

    def clear(self):
        self._store.clear()


device_cache = _DeviceCache()


@dataclass
class LoweredMotion:
    """An fm_motion struct plus the device buffers it points into."""
    struct: L.Motion
    keep: list = field(default_factory=list)

    @property
    def kind(self) -> int:
        return self.struct.kind


def _pod_term(obj, device) -> tuple[L.MotionTerm, list] | None:
    kind = None
    for klass in type(obj).__mro__:
        if klass.__name__ in _POD_NAMES:
            kind = _POD_NAMES[klass.__name__]
            break
    if kind is None:
        return None
    # The evaluation path must be the reference's own (Motion.py:165-172,
    # :240-254, :272-290); subclasses that override it are sampled instead.
    if not (_defined_by(obj, "__call__", {"POD"}) and
            _defined_by(obj, "_evaluate_trajectory", {"POD", "PODVelocity"}) and
            _defined_by(obj, "_evaluate_weights", {"POD"})):
        return None
    modes = getattr(obj, "_modes", None)
    pp = getattr(obj, "_pp_batch", None)
    if modes is None or pp is None or not hasattr(pp, "c") or not hasattr(pp, "x"):
        return None
    modes = np.asarray(modes)
    if modes.dtype != np.float32 or modes.ndim != 3 or modes.shape[1] != 3:
        return None
    if getattr(pp, "extrapolate", False) not in (True, False):
        return None  # 'periodic' extrapolation is not lowered
    weights = getattr(obj, "_weights", None)
    if weights is not None and np.asarray(weights).dtype != np.float32:
        return None
    c = np.asarray(pp.c)
    x = np.asarray(pp.x)
    if c.ndim != 3 or c.shape[2] != modes.shape[2] or np.iscomplexobj(c):
        return None
    ts_kind = num_kind(getattr(obj, "timeshift", 0.0))
    period = getattr(obj, "_period", None)
    p_kind = num_kind(period)
    if ts_kind in (None, L.FM_NUM_NONE) or p_kind is None:
        return None
    dev_modes = device_cache.get(modes, torch.float32, device)
    dev_c = device_cache.get(c, torch.float64, device)
    dev_x = device_cache.get(x, torch.float64, device)
    t = L.MotionTerm()
    t.kind = kind
    t.n_modes = modes.shape[2]
    t.modes = dev_modes.data_ptr()
    t.pp_c = dev_c.data_ptr()
    t.pp_x = dev_x.data_ptr()
    t.pp_k = c.shape[0]
    t.pp_intervals = c.shape[1]
    t.timeshift = float(np.asarray(obj.timeshift, dtype=np.float64))
    t.timeshift_kind = ts_kind
    t.period_kind = p_kind
    t.period = float(np.asarray(period, dtype=np.float64)) if period is not None else 0.0
    t.extrapolate = 1 if bool(pp.extrapolate) else 0
    return t, [dev_modes, dev_c, dev_x]


def _respiratory_term(obj, device) -> tuple[L.MotionTerm, list] | None:
    if not any(k.__name__ == "RespiratoryMotion" for k in type(obj).__mro__):
        return None
    if not (_defined_by(obj, "__call__", {"RespiratoryMotion"}) and
            _defined_by(obj, "_evaluate_motion", {"RespiratoryMotion"})):
        return None
    interp = getattr(obj, "interpolator", None)
    if interp is None or not hasattr(interp, "c") or not hasattr(interp, "x"):
        return None
    c = np.asarray(interp.c)
    if c.ndim != 2 or np.iscomplexobj(c):
        return None  # only scalar (1-D data) respiratory curves are lowered
    if getattr(interp, "extrapolate", True) not in (True, False):
        return None
    direction = np.asarray(getattr(obj, "direction"))
    if direction.dtype != np.float32 or direction.size != 3:
        return None
    ts_kind = num_kind(getattr(obj, "timeshift", 0.0))
    period = getattr(obj, "_period", None)
    p_kind = num_kind(period)
    if ts_kind in (None, L.FM_NUM_NONE) or p_kind is None:
        return None
    c3 = np.ascontiguousarray(c.reshape(c.shape[0], c.shape[1], 1))
    dev_c = torch.from_numpy(c3.astype(np.float64)).to(device)
    dev_x = torch.from_numpy(np.ascontiguousarray(interp.x, dtype=np.float64)).to(device)
    t = L.MotionTerm()
    t.kind = L.FM_TERM_RESPIRATORY
    t.n_modes = 1
    t.modes = None
    t.pp_c = dev_c.data_ptr()
    t.pp_x = dev_x.data_ptr()
    t.pp_k = c.shape[0]
    t.pp_intervals = c.shape[1]
    t.timeshift = float(np.asarray(obj.timeshift, dtype=np.float64))
    t.timeshift_kind = ts_kind
    t.period_kind = p_kind
    t.period = float(np.asarray(period, dtype=np.float64)) if period is not None else 0.0
    for i in range(3):
        t.direction[i] = float(direction.reshape(-1)[i])
    t.extrapolate = 1 if bool(interp.extrapolate) else 0
    return t, [dev_c, dev_x]


_SPEC_KINDS = {"modes": L.FM_TERM_POD, "velocity_modes": L.FM_TERM_POD_VELOCITY, "rigid": L.FM_TERM_RESPIRATORY}


def _spec_terms(obj, device) -> tuple[list, list] | None:
    """Terms of an object that states its own device form through
    fm_motion_terms() (feelmri_b200.motion.SplineMotion): each term's time
    is t + timeshift in float64, folded in float64 when it has a period."""
    specs = obj.fm_motion_terms()
    terms, keep = [], []
    for sp in specs:
        kind = _SPEC_KINDS.get(sp["kind"])
        if kind is None:
            return None
        c = np.ascontiguousarray(sp["coeffs"], np.float64)
        x = np.ascontiguousarray(sp["knots"], np.float64)
        dev_c = device_cache.get(c, torch.float64, device)
        dev_x = device_cache.get(x, torch.float64, device)
        t = L.MotionTerm()
        t.kind = kind
        t.pp_c = dev_c.data_ptr()
        t.pp_x = dev_x.data_ptr()
        t.pp_k = c.shape[0]
        t.pp_intervals = c.shape[1]
        t.timeshift = float(sp["timeshift"])
        t.timeshift_kind = L.FM_NUM_PYFLOAT
        t.period_kind = L.FM_NUM_NONE if sp["period"] is None else L.FM_NUM_F64
        t.period = 0.0 if sp["period"] is None else float(sp["period"])
        t.extrapolate = 1 if sp["extrapolate"] else 0
        if kind == L.FM_TERM_RESPIRATORY:
            t.n_modes = 1
            t.modes = None
            for i in range(3):
                t.direction[i] = float(np.float32(sp["direction"][i]))
            keep += [dev_c, dev_x]
        else:
            modes = sp["modes"]
            dev_modes = device_cache.get(modes, torch.float32, device)
            t.n_modes = modes.shape[2]
            t.modes = dev_modes.data_ptr()
            keep += [dev_modes, dev_c, dev_x]
        terms.append(t)
    return (terms, keep) if terms else None


def _terms(obj, device) -> tuple[list, list] | None:
    """Flattens a left-nested PODSum into terms added left to right."""
    if callable(getattr(obj, "fm_motion_terms", None)):
        return _spec_terms(obj, device)
    if any(k.__name__ == "PODSum" for k in type(obj).__mro__) and _defined_by(obj, "__call__", {"PODSum"}):
        left = _terms(obj.pod1, device)
        # pod1(t) + pod2(t): the right operand must be a single term so that
        # float32 additions happen in the same order as the reference's.
        right = _single(obj.pod2, device)
        if left is None or right is None:
            return None
        return left[0] + [right[0]], left[1] + right[1]
    one = _single(obj, device)
    if one is None:
        return None
    return [one[0]], one[1]


def _single(obj, device):
    return _pod_term(obj, device) or _respiratory_term(obj, device)


def term_timeshifts(obj) -> list | None:
    """(value, FM_NUM_* kind) of each term's .timeshift, in the order lower()
    lays the terms out (a left-nested PODSum left to right); None when a
    timeshift has a type lower() would refuse.  Reads only the timeshifts, so
    a block sequence can follow update_timeshift() without lowering again."""
    if callable(getattr(obj, "fm_motion_terms", None)):
        return [(float(sp["timeshift"]), L.FM_NUM_PYFLOAT) for sp in obj.fm_motion_terms()]
    if any(k.__name__ == "PODSum" for k in type(obj).__mro__) and _defined_by(obj, "__call__", {"PODSum"}):
        left = term_timeshifts(obj.pod1)
        right = term_timeshifts(obj.pod2)
        if left is None or right is None or len(right) != 1:
            return None
        return left + right
    ts = getattr(obj, "timeshift", 0.0)
    kind = num_kind(ts)
    if kind in (None, L.FM_NUM_NONE):
        return None
    return [(float(np.asarray(ts, dtype=np.float64)), kind)]


def lower(pod_trajectory, n_nodes: int, device: torch.device) -> LoweredMotion | None:
    """Returns the device descriptor of a motion callable, or None when the
    callable is not one this module can lower (the caller then samples it)."""
    m = L.Motion()
    if pod_trajectory is None:
        m.kind = L.FM_MOTION_NONE
        return LoweredMotion(m)
    res = _terms(pod_trajectory, device)
    if res is None or len(res[0]) > L.FM_MAX_MOTION_TERMS:
        return None
    terms, keep = res
    # POD modes must describe exactly the nodes of this call.
    for t, buf in zip(terms, _modes_buffers(terms, keep)):
        if buf is not None and buf.shape[0] != n_nodes:
            raise ValueError(f"pod_trajectory modes describe {buf.shape[0]} nodes, the call has {n_nodes}")
    m.kind = L.FM_MOTION_TERMS
    m.n_terms = len(terms)
    for i, t in enumerate(terms):
        m.terms[i] = t
    return LoweredMotion(m, keep)


def _modes_buffers(terms, keep):
    out = []
    k = 0
    for t in terms:
        if t.kind == L.FM_TERM_RESPIRATORY:
            out.append(None)
            k += 2
        else:
            out.append(keep[k])
            k += 3
    return out


def sample_table(pod_trajectory, times, n_nodes: int, np_dtype, device: torch.device) -> torch.Tensor:
    """Calls a generic motion callable at each time (as Python floats) and
    returns the stacked (len(times), N, 3) displacements on the device.  The
    reference converts each result to a C-contiguous array of the solver's
    real type (BlochSimulator.cpp:86, MRI.cpp:114) before reading N x 3 values."""
    out = torch.empty((len(times), n_nodes, 3), dtype=torch.float64 if np_dtype == np.float64 else torch.float32,
                      device=device)
    for i, t in enumerate(times):
        d = np.asarray(pod_trajectory(float(t)))
        d = np.ascontiguousarray(d, dtype=np_dtype)
        if d.size == 3 and n_nodes != 1:
            d = np.broadcast_to(d.reshape(1, 3), (n_nodes, 3))
        if d.size != n_nodes * 3:
            raise ValueError(f"pod_trajectory({t}) returned {d.shape}; expected ({n_nodes}, 3)")
        out[i].copy_(torch.from_numpy(np.ascontiguousarray(d.reshape(n_nodes, 3))))
    return out


def table_motion(table: torch.Tensor) -> LoweredMotion:
    m = L.Motion()
    m.kind = L.FM_MOTION_TABLE
    m.table = table.data_ptr()
    m.table_calls = table.shape[0]
    return LoweredMotion(m, [table])
