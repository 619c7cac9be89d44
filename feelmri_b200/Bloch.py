"""Sequence-level Bloch driver with the behaviour of BlochSolver.solve
(python/feelmri/Bloch.py:275-380), keeping the magnetisation on the GPU.

Per block (Bloch.py:332-368): the motion's timeshift is set to the block's
start, the block is discretised (times, rf, G; dt = diff(times, prepend=0)),
the fused sweep runs in its final-state form (fm_bloch_solve_f32), the final
state of blocks flagged store_magnetization is kept, and the state carried to
the next block is the final state, with Mxy replaced by 0 * Mxy after every
non-empty block (the reference's artificial spoiling).  solve(start, end)
returns (Mxy, Mz) of the stored blocks as (N, n_store) arrays and, like the
reference, updates initial_Mxy / initial_Mz so that a later solve(start=-2)
continues the sequence.

Blocks are workloads.Block objects (discretised arrays) or objects with the
reference SequenceBlock interface (_discretization(), __call__(times),
empty, store_magnetization, time_extent).
"""
from __future__ import annotations

import numpy as np
import torch

from . import ops
from ._motion import lower, sample_table, table_motion
from .BlochSimulator import bloch_call_times

__all__ = ["BlochSolver", "discretise"]


def _magnitude_ms(q):
    return q.m_as("ms") if hasattr(q, "m_as") else q


def discretise(block):
    """(times ms float64, rf complex64 (n_t,), G float32 (n_t, 3), t0 ms)."""
    if hasattr(block, "rf") and hasattr(block, "G") and hasattr(block, "times"):
        return (np.asarray(block.times, np.float64), np.asarray(block.rf, np.complex64).reshape(-1),
                np.asarray(block.G, np.float32), float(np.asarray(block.times)[0]))
    times = np.asarray(_magnitude_ms(block._discretization()), np.float64)
    rf_vals, G = block(times)
    rf = np.zeros(times.shape[0], np.complex64)
    rf[:] = rf_vals
    Gm = np.zeros((times.shape[0], 3), np.float32)
    for d in range(3):
        Gm[:, d] = G[d]
    t0 = float(_magnitude_ms(block.time_extent[0]))
    return times, rf, Gm, t0


class BlochSolver:
    def __init__(self, blocks, nodes, M0=1.0, T1=1000.0, T2=100.0, delta_B=0.0, gamma=267.522, pod_trajectory=None,
                 initial_Mxy=0.0, initial_Mz=None, device=None):
        self.blocks = list(blocks)
        nodes = np.asarray(nodes)
        N = nodes.shape[0]
        ones = np.ones((N, 1), np.float32)
        self.nodes = nodes
        self.M0 = M0
        self.gamma = gamma
        self.T1 = np.asarray(T1, np.float32).reshape(-1, 1) * ones if np.ndim(T1) else T1 * ones
        self.T2 = np.asarray(T2, np.float32).reshape(-1, 1) * ones if np.ndim(T2) else T2 * ones
        self.delta_B = np.asarray(delta_B, np.float32).reshape(-1, 1) * ones if np.ndim(delta_B) else delta_B * ones
        self.initial_Mxy = (np.asarray(initial_Mxy).reshape(-1, 1) * ones).astype(np.complex64)
        self.initial_Mz = (np.asarray(initial_Mz if initial_Mz is not None else M0).reshape(-1, 1) * ones).astype(
            np.float32)
        self.pod_trajectory = pod_trajectory
        self.device = device or ops.require_cuda()
        self._dev_static = None

    @property
    def n_nodes(self) -> int:
        return self.nodes.shape[0]

    def _static(self):
        if self._dev_static is None:
            dev = self.device

            def up(a, dt=torch.float32):
                return torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)
            self._dev_static = dict(r0=up(self.nodes.astype(np.float32)), T1=up(self.T1.reshape(-1)),
                                    T2=up(self.T2.reshape(-1)), dB=up(self.delta_B.reshape(-1)))
        return self._dev_static

    def solve(self, start: int = 0, end: int | None = None):
        if start < 0:
            start += len(self.blocks)
        if end is None:
            end = len(self.blocks)
        blocks = self.blocks[start:end]
        N = self.n_nodes
        dev = self.device
        st = self._static()
        store = [i for i, b in enumerate(blocks) if b.store_magnetization]
        out_m = torch.zeros((max(len(store), 1), N), dtype=torch.complex64, device=dev)
        out_z = torch.zeros((max(len(store), 1), N), dtype=torch.float32, device=dev)
        m = torch.from_numpy(self.initial_Mxy.reshape(-1).copy()).to(dev)
        z = torch.from_numpy(self.initial_Mz.reshape(-1).copy()).to(dev)
        for i, block in enumerate(blocks):
            times, rf, G, t0 = discretise(block)
            if self.pod_trajectory is not None:
                self.pod_trajectory.update_timeshift(t0)
            dt = np.diff(times, prepend=0).astype(np.float32)
            inp = ops.BlochInputs(r0=st["r0"], T1=st["T1"], T2=st["T2"], delta_B=st["dB"], M0=self.M0,
                                  gamma=self.gamma, rf=torch.from_numpy(rf).to(dev),
                                  G=torch.from_numpy(np.ascontiguousarray(G)).to(dev),
                                  dt=torch.from_numpy(dt).to(dev), Mxy0=m, Mz0=z)
            motion = lower(self.pod_trajectory, N, dev)
            if motion is None:
                motion = table_motion(sample_table(self.pod_trajectory, bloch_call_times(dt), N, np.float32, dev))
            k = store.index(i) if i in store else None
            empty = bool(getattr(block, "empty", False))
            # stored final state -> output column; carried state -> m / z in
            # place (0 * Mxy after a non-empty block, Bloch.py:363-368)
            fin_m = out_m[k] if k is not None else (m if empty else None)
            fin_z = out_z[k] if k is not None else z
            ops.bloch_solve(inp, motion, history=False, Mxy_final=fin_m, Mz_final=fin_z,
                            Mxy_carry=None if empty else m, allocate_final=False)
            if k is not None:
                z.copy_(fin_z)
                if empty:
                    m.copy_(fin_m)
        self.initial_Mxy[:, 0] = m.cpu().numpy()
        self.initial_Mz[:, 0] = z.cpu().numpy()
        if not store:
            return np.zeros((N, 0), np.complex64), np.zeros((N, 0), np.float32)
        return out_m.cpu().numpy().T, out_z.cpu().numpy().T
