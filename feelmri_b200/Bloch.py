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

The constructor takes the reference's arguments in the reference's order
(Bloch.py:276-297): a Sequence (anything with .blocks; a plain list of blocks
also works), a FEMPhantom (anything with .local_nodes; an (N, 3) array also
works), a Scanner (its .gamma, a pint quantity converted to rad/(ms mT), or a
plain number; None means the reference's default Scanner, gamma =
42.58e6 * 2 pi rad Hz/T), M0, T1 and T2 (pint quantities converted to ms, or
numbers in ms), delta_B, pod_trajectory, initial_Mxy and initial_Mz.  The
blocks are read from the sequence at each solve(), as the reference does.
Blocks are workloads.Block objects (discretised arrays) or objects with the
reference SequenceBlock interface (_discretization(), __call__(times),
empty, store_magnetization, time_extent).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from . import ops
from ._motion import lower, sample_table, table_motion, term_timeshifts
from .BlochSimulator import bloch_call_times

__all__ = ["BlochSolver", "discretise", "DEFAULT_GAMMA"]

# the reference Scanner's gamma, 42.58e6 * 2 pi rad Hz/T, in rad/(ms mT) (MRObjects.py:38-40)
DEFAULT_GAMMA = 42.58e6 * 2 * np.pi * 1e-6


def _magnitude_ms(q):
    return q.m_as("ms") if hasattr(q, "m_as") else q


def _gamma_of(scanner) -> float:
    """rad/(ms mT) from a Scanner-like object, a quantity or a number."""
    if scanner is None:
        return DEFAULT_GAMMA
    g = getattr(scanner, "gamma", scanner)
    if hasattr(g, "m_as"):
        return float(g.m_as("rad/ms/mT"))
    return float(g)


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


_STATE = {"initial_Mxy": (np.complex64, torch.complex64), "initial_Mz": (np.float32, torch.float32)}
_PARAMS = ("T1", "T2", "delta_B")


class BlochSolver:
    """Per-node parameters and the carried state live on the device.

    T1, T2, delta_B, initial_Mxy and initial_Mz read as the reference's (N, 1)
    host arrays (Bloch.py:285-293), built on first access.  Values are taken
    at construction: scalars are filled on the device, arrays uploaded once.
    The carried state stays on the GPU between solves.  Once a host array has
    been read it is the one the next solve starts from, so in-place edits take
    effect, and each solve writes the carried state back into initial_Mxy /
    initial_Mz in place, as the reference does (Bloch.py:363-368).  Arrays
    that were never read are never copied to the host."""

    def __init__(self, sequence, phantom, scanner=None, M0=1.0, T1=1000.0, T2=100.0, delta_B=0.0,
                 pod_trajectory=None, initial_Mxy=0.0, initial_Mz=None, *, gamma=None, device=None):
        self.sequence = sequence
        self.phantom = phantom
        self.scanner = scanner
        self.nodes = np.asarray(getattr(phantom, "local_nodes", phantom))
        if self.nodes.ndim != 2 or self.nodes.shape[1] != 3:
            raise ValueError(f"BlochSolver: phantom nodes must be (N, 3), got {self.nodes.shape}")
        self.M0 = M0
        self.gamma = _gamma_of(scanner) if gamma is None else float(gamma)
        self.pod_trajectory = pod_trajectory
        self.device = device or ops.require_cuda()
        self._given = {"T1": _magnitude_ms(T1), "T2": _magnitude_ms(T2), "delta_B": delta_B,
                       "initial_Mxy": initial_Mxy, "initial_Mz": initial_Mz if initial_Mz is not None else M0}
        self._host: dict[str, np.ndarray] = {}
        self._dev: dict[str, torch.Tensor] = {}
        # nodes and every per-node array go up in one transfer; single values are filled
        pending = [("nodes", np.asarray(self.nodes, np.float32), torch.float32)]
        for name in (*_PARAMS, *_STATE):
            snap = self._snapshot(name)
            if isinstance(snap, torch.Tensor):
                self._dev[name] = snap
            else:
                pending.append((name, snap, _STATE.get(name, (None, torch.float32))[1]))
        dev_arrays = ops.upload_many([(a, dt) for _, a, dt in pending], self.device)
        self._dev_nodes = dev_arrays[0]
        for (name, _, _), t in zip(pending[1:], dev_arrays[1:]):
            self._dev[name] = t

    @property
    def n_nodes(self) -> int:
        return self.nodes.shape[0]

    @property
    def blocks(self) -> list:
        """The sequence's blocks, read afresh (blocks added later are seen)."""
        return list(getattr(self.sequence, "blocks", self.sequence))

    def _construct(self, name: str) -> np.ndarray:
        """The (N, 1) host array the reference builds (Bloch.py:285-293)."""
        ones = np.ones((self.n_nodes, 1), np.float32)
        v = self._given[name]
        if name in _STATE:
            return (np.asarray(v).reshape(-1, 1) * ones).astype(_STATE[name][0])
        return np.asarray(v, np.float32).reshape(-1, 1) * ones if np.ndim(v) else v * ones

    def _snapshot(self, name: str):
        """The constructed value as an (N,) device fill for one value, else as
        the (N,) host array to upload (an array of N parameter values is taken
        as given: multiplying it by ones leaves it unchanged)."""
        N = self.n_nodes
        np_t, torch_t = _STATE.get(name, (np.float32, torch.float32))
        v = self._given[name]
        if np.size(v) == 1:
            if name in _STATE:
                one = (np.asarray(v).reshape(-1, 1) * np.ones((1, 1), np.float32)).astype(np_t)
            elif np.ndim(v):
                one = np.asarray(v, np.float32)
            else:
                one = np.asarray(v * np.ones((1, 1), np.float32))
            return torch.full((N,), one.reshape(-1)[0].item(), dtype=torch_t, device=self.device)
        if name not in _STATE and np.size(v) == N:
            flat = np.asarray(v, np.float32).reshape(-1)
        else:
            flat = self._construct(name).reshape(-1)
        if flat.size != N:
            raise ValueError(f"BlochSolver: {flat.size} values for {N} nodes")
        return flat.astype(np_t, copy=False)

    def _upload(self, flat: np.ndarray, np_t) -> torch.Tensor:
        if flat.size != self.n_nodes:
            raise ValueError(f"BlochSolver: {flat.size} values for {self.n_nodes} nodes")
        return torch.from_numpy(np.ascontiguousarray(flat.astype(np_t, copy=False))).to(self.device)

    def _host_array(self, name: str) -> np.ndarray:
        if name not in self._host:
            if name in _STATE:
                self._host[name] = self._dev[name].cpu().numpy().reshape(self.n_nodes, 1)
            else:
                self._host[name] = self._construct(name)
        return self._host[name]

    def _set_host(self, name: str, value) -> None:
        self._host[name] = np.asarray(value)

    T1 = property(lambda self: self._host_array("T1"), lambda self, v: self._set_host("T1", v))
    T2 = property(lambda self: self._host_array("T2"), lambda self, v: self._set_host("T2", v))
    delta_B = property(lambda self: self._host_array("delta_B"), lambda self, v: self._set_host("delta_B", v))
    initial_Mxy = property(lambda self: self._host_array("initial_Mxy"),
                           lambda self, v: self._set_host("initial_Mxy", v))
    initial_Mz = property(lambda self: self._host_array("initial_Mz"),
                          lambda self, v: self._set_host("initial_Mz", v))

    def _device_array(self, name: str) -> torch.Tensor:
        """The value a solve starts from: the host array when one has been
        handed out (it may have been edited), else the device copy."""
        if name in self._host:
            self._dev[name] = self._upload(np.asarray(self._host[name]).reshape(-1),
                                           _STATE.get(name, (np.float32,))[0])
        return self._dev[name]

    def solve(self, start: int = 0, end: int | None = None):
        if start < 0:
            start += len(self.blocks)
        if end is None:
            end = len(self.blocks)
        blocks = self.blocks[start:end]
        N = self.n_nodes
        dev = self.device
        r0 = self._dev_nodes
        T1, T2, dB = (self._device_array(n) for n in _PARAMS)
        store = [i for i, b in enumerate(blocks) if b.store_magnetization]
        out_m = torch.zeros((max(len(store), 1), N), dtype=torch.complex64, device=dev)
        out_z = torch.zeros((max(len(store), 1), N), dtype=torch.float32, device=dev)
        m = self._device_array("initial_Mxy")
        z = self._device_array("initial_Mz")
        if blocks and lower(self.pod_trajectory, N, dev) is not None:
            self._solve_sequence(blocks, store, r0, T1, T2, dB, m, z, out_m, out_z)
        else:
            self._solve_blocks(blocks, store, r0, T1, T2, dB, m, z, out_m, out_z)
        for name, t in (("initial_Mxy", m), ("initial_Mz", z)):
            if name in self._host:  # handed out: updated in place, as the reference does
                host = self._host[name]
                if host.ndim == 2:
                    host[:, 0] = t.cpu().numpy()
                else:
                    host[...] = t.cpu().numpy().reshape(host.shape)
        if not store:
            return np.zeros((N, 0), np.complex64), np.zeros((N, 0), np.float32)
        host_m, host_z = ops.to_host(out_m, out_z)
        return host_m.T, host_z.T

    def _solve_sequence(self, blocks, store, r0, T1, T2, dB, m, z, out_m, out_z):
        """Every block in one sweep (fm_bloch_sequence_f32).  The motion is
        lowered per block after update_timeshift(t0), as the block loop does;
        the lowered descriptors differ only in their timeshifts."""
        N = self.n_nodes
        dev = self.device
        seq, rfs, Gs, dts = [], [], [], []
        motion = None
        for i, block in enumerate(blocks):
            times, rf, G, t0 = discretise(block)
            if self.pod_trajectory is not None:
                self.pod_trajectory.update_timeshift(t0)
            if motion is None:
                motion = lower(self.pod_trajectory, N, dev)
                if motion is None:  # the callable no longer lowers: run block by block
                    return self._solve_blocks(blocks, store, r0, T1, T2, dB, m, z, out_m, out_z)
            shifts = ()
            if motion.struct.kind == L.FM_MOTION_TERMS:
                ts = term_timeshifts(self.pod_trajectory)
                if ts is None or len(ts) != motion.struct.n_terms:
                    return self._solve_blocks(blocks, store, r0, T1, T2, dB, m, z, out_m, out_z)
                shifts = tuple(ts)
            seq.append(ops.SequenceBlock(n_time=times.shape[0], empty=bool(getattr(block, "empty", False)),
                                         store=store.index(i) if i in store else -1, timeshifts=shifts))
            rfs.append(rf)
            Gs.append(np.ascontiguousarray(G, np.float32).reshape(-1, 3))
            dts.append(np.diff(times, prepend=0).astype(np.float32))
        rf, G, dt = ops.upload_many([(np.concatenate(rfs), torch.complex64), (np.concatenate(Gs), torch.float32),
                                     (np.concatenate(dts), torch.float32)], dev)
        ops.bloch_sequence(r0, T1, T2, dB, self.M0, self.gamma, seq, rf, G, dt, m, z, motion, out_m, out_z,
                           Mxy_carry=m, Mz_carry=z)

    def _solve_blocks(self, blocks, store, r0, T1, T2, dB, m, z, out_m, out_z):
        """Block by block (a motion that is sampled on the host)."""
        N = self.n_nodes
        dev = self.device
        for i, block in enumerate(blocks):
            times, rf, G, t0 = discretise(block)
            if self.pod_trajectory is not None:
                self.pod_trajectory.update_timeshift(t0)
            dt = np.diff(times, prepend=0).astype(np.float32)
            d_rf, d_G, d_dt = ops.upload_many([(rf, torch.complex64), (G, torch.float32), (dt, torch.float32)], dev)
            inp = ops.BlochInputs(r0=r0, T1=T1, T2=T2, delta_B=dB, M0=self.M0, gamma=self.gamma, rf=d_rf, G=d_G,
                                  dt=d_dt, Mxy0=m, Mz0=z)
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
