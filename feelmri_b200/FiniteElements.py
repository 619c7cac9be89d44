"""P1 tetrahedral element and quadrature without basix.

Same interface as python/feelmri/FiniteElements.py:30-99 (FiniteElement with
.dimension and .tabulate(derivative_order, points); QuadratureRule with
.points and .weights), restricted to what the hot path uses: the degree-1
Lagrange tetrahedron and the order-1/2 tetrahedron rules.  Values are cast to
`dtype` (float32 by default) exactly as the reference's wrappers cast basix's
output (FiniteElements.py:35, :68, :74, :98-99).

Basis (reference cell with vertices (0,0,0), (1,0,0), (0,1,0), (0,0,1)):
  S0 = 1 - x - y - z, S1 = x, S2 = y, S3 = z, with constant gradients.
Quadrature: order 1 is the centroid with weight 1/6; order 2 is the symmetric
4-point rule with a = (5 - sqrt 5)/20, b = (5 + 3 sqrt 5)/20, weights 1/24.
These are the published rules of the stated degree; basix is absent here, so
their point order and float32 rounding are not checked against it.
"""
from __future__ import annotations

import numpy as np

__all__ = ["FiniteElement", "QuadratureRule"]

_GRAD = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


class FiniteElement:
    def __init__(self, family="P", cell_type="tetrahedron", degree=1, variant="equispaced", dtype=np.float32):
        if family != "P" or cell_type != "tetrahedron" or degree != 1:
            raise NotImplementedError("only the P1 tetrahedron is provided")
        self.family = family
        self.cell_type = cell_type
        self.degree = degree
        self.variant = variant
        self.dtype = dtype
        self.dimension = 4

    def tabulate(self, derivative_order, points):
        """(n_derivs, n_points, 4, 1): values, then first derivatives."""
        pts = np.atleast_2d(np.asarray(points, dtype=np.float64))
        n = pts.shape[0]
        nd = 1 if derivative_order == 0 else 4
        if derivative_order not in (0, 1):
            raise NotImplementedError("derivatives above first order vanish for P1 and are not tabulated")
        out = np.zeros((nd, n, 4, 1), dtype=np.float64)
        x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
        out[0, :, 0, 0] = 1.0 - x - y - z
        out[0, :, 1, 0] = x
        out[0, :, 2, 0] = y
        out[0, :, 3, 0] = z
        if nd == 4:
            for d in range(3):
                out[d + 1, :, :, 0] = _GRAD[:, d][None, :]
        return out.astype(self.dtype)


class QuadratureRule:
    def __init__(self, cell_type="tetrahedron", order=2, rule="default", dtype=np.float32):
        if cell_type != "tetrahedron":
            raise NotImplementedError("only tetrahedron rules are provided")
        if order <= 1:
            pts = np.array([[0.25, 0.25, 0.25]])
            w = np.array([1.0 / 6.0])
        elif order == 2:
            a = (5.0 - np.sqrt(5.0)) / 20.0
            b = (5.0 + 3.0 * np.sqrt(5.0)) / 20.0
            pts = np.array([[a, a, a], [b, a, a], [a, b, a], [a, a, b]])
            w = np.full(4, 1.0 / 24.0)
        else:
            raise NotImplementedError("tetrahedron rules above order 2 are not provided")
        self.cell_type = cell_type
        self.order = order
        self.rule = rule
        self.points = pts.astype(dtype)
        self.weights = w.astype(dtype)
