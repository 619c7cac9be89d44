"""Drop-in for the reference module `feelmri.POD`.

tensordot_modes_weights(modes, weights) keeps the reference's two
`noconvert` overloads (cpp/feelmri/POD.h:16-24): both arguments must be
C-contiguous numpy arrays of the same dtype, float32 or float64, otherwise
TypeError.  Returns out[p, c] = sum_m modes[p, c, m] * weights[m] as a new
(P, C) array, computed on the GPU (fm_pod_tensordot_*).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _pybind as pb
from . import ops

__all__ = ["tensordot_modes_weights"]


def _exact(obj, dtype) -> bool:
    return isinstance(obj, np.ndarray) and obj.dtype == dtype and obj.flags.c_contiguous


def tensordot_modes_weights(modes, weights):
    """(P, C, M) . (M,) -> (P, C)."""
    for dtype, tdtype in ((np.float32, torch.float32), (np.float64, torch.float64)):
        if _exact(modes, dtype) and _exact(weights, dtype):
            break
    else:
        raise pb.no_overload("tensordot_modes_weights", (modes, weights))
    if modes.ndim != 3:
        raise ValueError(f"tensordot_modes_weights: modes must be (P, C, M); got {modes.shape}")
    if weights.ndim != 1 or weights.shape[0] != modes.shape[2]:
        raise ValueError(f"tensordot_modes_weights: weights {weights.shape} do not match modes {modes.shape}")
    dev = ops.require_cuda()
    m = torch.from_numpy(modes).to(dev)
    w = torch.from_numpy(weights).to(dev)
    return ops.to_host(ops.tensordot_modes_weights(m, w))
