"""Request loop for simulations: admission by HBM footprint, device-resident
state, overlapping execution and latency statistics.

A request is one simulation: a mesh with tissue parameters, the imaging
blocks of a sequence, a k-space trajectory, receive coils and a number of
cardiac frames (with optional motion).  Once admitted, everything a request
needs stays on the GPU until it completes:

* the mesh, tissue arrays, lumped P1 mass weights (assembled on the device)
  and coil maps;
* the magnetisation (Mxy, Mz), carried from block to block and frame to
  frame by the fused Bloch sweep;
* the Signal workspace, reused frame after frame.

Serving is continuous: a dispatcher admits arriving requests whenever a
slot is free and the HBM budget holds their footprint, and every slot runs
its request's frames on its own CUDA stream.  Requests therefore overlap on
the device, and a new one does not wait for the others to finish.  Each
request's result depends only on its own inputs: its kernels, tile shapes and
reduction orders do not depend on what else runs, so it is the same alone and
in a mix.

The reference has no serving mode (its examples loop over frames in Python,
e.g. examples/phase_contrast.py:198-207); this module is new.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import ops
from ._motion import lower
from .workloads import GAMMA, Block, Mesh, Trajectory

__all__ = ["Request", "Simulation", "Server", "latency_stats"]


@dataclass
class Request:
    rid: int
    mesh: Mesh
    T1: np.ndarray            # (N,) ms
    T2: np.ndarray            # (N,) ms
    phi: np.ndarray           # (N,) rad/ms off-resonance
    blocks: list[Block]       # sequence blocks simulated before each frame's readout
    traj: Trajectory
    coils: np.ndarray         # (N, C) complex64 receive sensitivities
    frames: int = 1
    frame_ms: float = 40.0    # time between frames (motion timeshift)
    pod: object = None        # motion callable (reference classes are lowered to the GPU)
    precision: str = "bf16x3"
    arrival: float = 0.0      # seconds after the start of the run

    @property
    def n_nodes(self) -> int:
        return self.mesh.n_nodes

    @property
    def work(self) -> float:
        """node*k-samples of the whole request."""
        return float(self.n_nodes) * self.traj.n_samples * self.frames


def footprint_bytes(req: Request) -> int:
    """Device bytes a request holds while admitted (state, inputs, outputs and
    the Signal workspace), estimated from its sizes."""
    N, S, C = req.n_nodes, req.traj.n_samples, req.coils.shape[1]
    E = req.mesh.elems.shape[0]
    state = N * (12 + 4 * 4 + 8 + 4 + 8 * C * 2)           # nodes, tissue, mass, Mxy/Mz, coils, Mxy columns
    traj = S * 16 + S * C * 8                              # k, t, one output frame
    mass_setup = E * 16 * 32                               # assembly triplets (transient)
    signal_ws = N * C * 8 + S * 64 + 16 * S * C * 8
    return int(state + traj + max(mass_setup, signal_ws) + (64 << 20))


class Simulation:
    """Device-resident state of one admitted request, bound to one stream."""

    def __init__(self, req: Request, device: torch.device, stream: torch.cuda.Stream):
        from .Assemble import mass_lumped
        from .FiniteElements import FiniteElement, QuadratureRule
        self.req = req
        self.device = device
        self.stream = stream
        N = req.n_nodes
        with torch.cuda.stream(stream):
            def up(a, dt=torch.float32):
                return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dt, non_blocking=True)
            w = mass_lumped(req.mesh.elems, req.mesh.nodes, FiniteElement(), QuadratureRule(order=2))
            self.r0 = up(req.mesh.nodes.astype(np.float32))
            self.T1, self.T2 = up(req.T1), up(req.T2)
            self.dB = torch.zeros(N, dtype=torch.float32, device=device)
            self.phi = up(req.phi)
            self.coils = up(req.coils, torch.complex64)
            self.blocks = [(up(b.rf, torch.complex64), up(b.G), up(b.dt.astype(np.float32)), b.t0, b.empty)
                           for b in req.blocks]
            self.M = ops.SparseCSC((N, N), up(np.arange(N + 1, dtype=np.int32), torch.int32),
                                   up(np.arange(N, dtype=np.int32), torch.int32), up(w.astype(np.float32)))
            t = req.traj
            self.kx, self.ky, self.kz, self.t = up(t.kx), up(t.ky), up(t.kz), up(t.t)
            self.Mxy = torch.zeros(N, dtype=torch.complex64, device=device)
            self.Mz = torch.ones(N, dtype=torch.float32, device=device)
            self.cols = torch.empty((N, req.coils.shape[1]), dtype=torch.complex64, device=device)
            self.out = torch.empty((*t.shape, req.coils.shape[1]), dtype=torch.complex64, device=device)
            self.sig = ops.SignalInputs(M=self.M, kx=self.kx, ky=self.ky, kz=self.kz, t=self.t, r0=self.r0,
                                        phi=self.phi, T2=self.T2, Mxy=self.cols)
            # the workspace holds per-time motion weights: size it with the request's motion
            a = ops.signal_args(self.sig, lower(req.pod, N, device), req.precision, self.out)
            self.ws = torch.empty(ops.signal_workspace_bytes(a, req.precision), dtype=torch.uint8, device=device)
        self.kspace = np.empty((req.frames, *t.shape, req.coils.shape[1]), np.complex64)

    def run(self) -> np.ndarray:
        """All frames.  Per frame the sequence blocks run with the state carried
        (Mxy spoiled after non-empty blocks, as BlochSolver does); the last
        block's final, unspoiled Mxy is read out through every coil."""
        req = self.req
        N = req.n_nodes
        readout = torch.empty(N, dtype=torch.complex64, device=self.device)
        pinned = torch.empty(self.out.shape, dtype=torch.complex64, pin_memory=True)
        with torch.cuda.stream(self.stream):
            for f in range(req.frames):
                for bi, (rf, G, dt, t0, empty) in enumerate(self.blocks):
                    last = bi == len(self.blocks) - 1
                    if req.pod is not None:
                        req.pod.update_timeshift(f * req.frame_ms + t0)
                    inp = ops.BlochInputs(r0=self.r0, T1=self.T1, T2=self.T2, delta_B=self.dB, M0=1.0, gamma=GAMMA,
                                          rf=rf, G=G, dt=dt, Mxy0=self.Mxy, Mz0=self.Mz)
                    final = self.Mxy if empty else (readout if last else None)
                    ops.bloch_solve(inp, lower(req.pod, N, self.device), history=False, Mxy_final=final,
                                    Mz_final=self.Mz, Mxy_carry=None if empty else self.Mxy, allocate_final=False)
                    if last:
                        src = self.Mxy if empty else readout
                ops.coil_expand(src, self.coils, out=self.cols)
                if req.pod is not None:
                    req.pod.update_timeshift(f * req.frame_ms)
                motion = lower(req.pod, N, self.device)
                ops.signal(self.sig, motion, req.precision, out=self.out, sync=False, ws=self.ws)
                ops.signal_status(self.sig, motion, req.precision, self.out, self.ws)
                pinned.copy_(self.out, non_blocking=True)
                self.stream.synchronize()
                self.kspace[f] = pinned.numpy()
        return self.kspace


def latency_stats(latencies: list[float]) -> dict:
    lat = np.sort(np.asarray(latencies, dtype=np.float64))
    if lat.size == 0:
        return {"p50_s": None, "p99_s": None, "n": 0}
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max()), "n": int(lat.size)}


@dataclass
class Served:
    req: Request
    arrival: float
    admitted: float = 0.0
    finished: float = 0.0
    kspace: np.ndarray | None = None
    error: str | None = None


@dataclass
class Server:
    """Continuous-batching request loop on one GPU.

    slots:       requests that may run at the same time (one stream each);
    hbm_budget:  bytes of device memory the admitted requests may hold."""
    device: torch.device = None
    slots: int = 4
    hbm_budget: int = 0
    results: list = field(default_factory=list)

    def __post_init__(self):
        self.device = self.device or ops.require_cuda()
        if not self.hbm_budget:
            free, _ = torch.cuda.mem_get_info(self.device)
            self.hbm_budget = int(free * 0.8)
        self._lock = threading.Condition()
        self._in_use = 0
        self._running = 0
        self._streams = [torch.cuda.Stream(device=self.device) for _ in range(self.slots)]
        self._free_streams = list(range(self.slots))

    def _admit(self, need: int) -> int | None:
        if self._running >= self.slots or not self._free_streams:
            return None
        if self._in_use + need > self.hbm_budget and self._running > 0:
            return None
        self._in_use += need
        self._running += 1
        return self._free_streams.pop()

    def _release(self, need: int, slot: int):
        with self._lock:
            self._in_use -= need
            self._running -= 1
            self._free_streams.append(slot)
            self._lock.notify_all()

    def _worker(self, item: Served, slot: int, need: int, t0: float):
        try:
            torch.cuda.set_device(self.device)
            sim = Simulation(item.req, self.device, self._streams[slot])
            item.kspace = sim.run()
        except Exception as exc:  # noqa: BLE001 - the request fails, the server goes on
            item.error = f"{type(exc).__name__}: {exc}"
        finally:
            item.finished = time.perf_counter() - t0
            self._release(need, slot)

    def serve(self, requests: list[Request], realtime: bool = True) -> list[Served]:
        """Runs the requests, each arriving at req.arrival seconds (when
        realtime) and admitted as soon as a slot and memory allow; returns one
        record per request with its times and k-space."""
        order = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        items = [Served(r, r.arrival) for r in order]
        threads = []
        pending = list(items)
        while pending:
            item = pending[0]
            now = time.perf_counter() - t0
            if realtime and now < item.arrival:
                time.sleep(min(item.arrival - now, 0.01))
                continue
            need = footprint_bytes(item.req)
            with self._lock:
                slot = self._admit(need)
                while slot is None:
                    self._lock.wait(timeout=0.05)
                    slot = self._admit(need)
            item.admitted = time.perf_counter() - t0
            pending.pop(0)
            th = threading.Thread(target=self._worker, args=(item, slot, need, t0), daemon=True)
            th.start()
            threads.append(th)
        for th in threads:
            th.join()
        self.results.extend(items)
        return items

    @staticmethod
    def summary(items: list[Served], wall_s: float | None = None) -> dict:
        done = [it for it in items if it.error is None]
        lat = [it.finished - it.arrival for it in done]
        work = sum(it.req.work for it in done)
        span = wall_s if wall_s is not None else (max((it.finished for it in done), default=0.0) -
                                                  min((it.arrival for it in done), default=0.0))
        out = latency_stats(lat)
        out.update({"requests": len(items), "failed": len(items) - len(done),
                    "throughput_node_samples_per_s": work / span if span > 0 else None, "span_s": span})
        return out
