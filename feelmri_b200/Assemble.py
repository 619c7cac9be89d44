"""Drop-in for the reference module `feelmri.Assemble`.

MassAssemble(elems, nodes, finite_element, quadrature_rule) keeps the
reference's overloads (cpp/feelmri/Assemble.h:26-38): float first, then
double.  The double overload runs only for int32 `elems` with float64
`nodes`; any conversion (e.g. int64 elems) selects float, as pybind11's
second pass does.  Returns a scipy.sparse.csc_matrix (N, N) with the sparsity
and duplicate-summation order of Eigen's setFromTriplets.

The reference calls finite_element.tabulate(1, qpoint) once per element and
quadrature point (Assemble.cpp:24, :69-73); the values do not depend on the
element, so they are tabulated once per quadrature point here and the whole
assembly runs on the GPU (fm_mass_assemble).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from . import _pybind as pb
from . import ops

__all__ = ["MassAssemble", "tabulate_at_quadrature", "mass_lumped"]


def tabulate_at_quadrature(finite_element, quadrature_rule, T):
    """(qweights (Q,), table (Q, 4, nb)) in dtype T, read through the same
    casts the reference applies (Assemble.cpp:24-33, :95-97)."""
    qpoints = pb.dense(quadrature_rule.points, T, True)
    qweights = pb.dense(quadrature_rule.weights, T, True, vector=True)
    nb = int(finite_element.dimension)
    tab = np.empty((qpoints.shape[0], 4, nb), dtype=T)
    for q in range(qpoints.shape[0]):
        vals = np.asarray(finite_element.tabulate(1, np.ascontiguousarray(qpoints[q:q + 1, :]))).astype(T)
        if vals.ndim != 4 or vals.shape[0] < 4 or vals.shape[2] != nb:
            raise ValueError(f"tabulate(1, point) returned shape {vals.shape}; expected (4, 1, {nb}, 1)")
        tab[q] = vals[:4, 0, :, 0]
    return np.ascontiguousarray(qweights), tab


def _load(args, T, convert):
    elems, nodes, fe, qr = args
    return dict(elems=pb.dense(elems, np.int32, convert), nodes=pb.dense(nodes, T, convert), fe=fe, qr=qr, T=T)


def _device_inputs(elems, nodes, fe, qr, T):
    if elems.ndim != 2 or elems.shape[0] == 0:
        raise ValueError("MassAssemble: elems must be a non-empty (E, nb) array (the reference reads elems.row(0))")
    nb = int(fe.dimension)
    if elems.shape[1] != nb:
        raise ValueError(f"MassAssemble: elements have {elems.shape[1]} nodes, the finite element {nb} dofs")
    if nodes.shape[1] != 3:
        raise ValueError(f"MassAssemble: nodes must be (N, 3); got {nodes.shape}")
    qw, tab = tabulate_at_quadrature(fe, qr, T)
    dev = ops.require_cuda()
    real = torch.float64 if T == np.float64 else torch.float32
    return dev, (torch.from_numpy(np.ascontiguousarray(elems, dtype=np.int32)).to(dev),
                 torch.from_numpy(np.ascontiguousarray(nodes)).to(device=dev, dtype=real),
                 torch.from_numpy(qw).to(device=dev, dtype=real),
                 torch.from_numpy(np.ascontiguousarray(tab)).to(device=dev, dtype=real))


def MassAssemble(elems, nodes, finite_element, quadrature_rule):
    """Consistent finite-element mass matrix as a CSC matrix (see module docstring)."""
    args = (elems, nodes, finite_element, quadrature_rule)
    for convert in (False, True):
        for T in (np.float32, np.float64):
            try:
                a = _load(args, T, convert)
            except pb.NoMatch:
                continue
            dev, dargs = _device_inputs(a["elems"], a["nodes"], finite_element, quadrature_rule, T)
            indptr, indices, data = ops.mass_assemble(*dargs)
            N = a["nodes"].shape[0]
            return sp.csc_matrix((data.cpu().numpy(), indices.cpu().numpy(), indptr.cpu().numpy()), shape=(N, N))
    raise pb.no_overload("MassAssemble", args)


def mass_lumped(elems, nodes, finite_element, quadrature_rule) -> np.ndarray:
    """Row sums of MassAssemble(...) as FEMPhantom.mass_matrix(lumped=True)
    forms them (python/feelmri/Phantom.py:395-398), computed on the GPU."""
    args = (elems, nodes, finite_element, quadrature_rule)
    for convert in (False, True):
        for T in (np.float32, np.float64):
            try:
                a = _load(args, T, convert)
            except pb.NoMatch:
                continue
            dev, dargs = _device_inputs(a["elems"], a["nodes"], finite_element, quadrature_rule, T)
            return ops.mass_lumped(*dargs).cpu().numpy()
    raise pb.no_overload("mass_lumped", args)
