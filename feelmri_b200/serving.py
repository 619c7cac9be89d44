"""Many simulations on one GPU: batched frames, continuous admission and
latency statistics.

A request is one simulation: a mesh with tissue parameters, the imaging
blocks of a sequence, a k-space trajectory, receive coils and a number of
cardiac frames (with optional motion).  Once admitted, everything a request
needs stays on the GPU until it completes:

* the mesh, tissue arrays, lumped P1 mass weights (assembled on the device)
  and coil maps, uploaded through one pinned staging buffer;
* the magnetisation (Mxy, Mz), carried from block to block and frame to
  frame by the fused Bloch sweep;
* the k-space output buffer, reused frame after frame.

Execution is batched by frame.  One *iteration* advances every admitted
request by one frame: each request's Bloch blocks and coil expansion, then
ONE persistent tensor-core launch (fm_signal_batch_enqueue) that contracts
the Signal of all of them together -- the requests' work units share the
SMs inside that launch -- then one copy of every output to pinned host
memory.  Requests that arrive while an iteration runs are set up (upload,
mass assembly) on a side stream and join the next iteration, as far as the
slot count and the HBM budget allow; requests whose last frame is done leave.
This is continuous batching at frame granularity.

A request's result depends only on its own inputs: its Signal work units,
their node splits and the reduction order are fixed by the request and the
server's fixed tuning (ops.Tuning), never by the other requests in the
launch, so it is the same alone and in any mix, bit for bit.

``simulate_batch`` runs one frame of many simulations from host arrays to
host arrays through the same machinery (the batched configuration's public
call).  The reference has no serving or batching mode (its examples loop
over phantoms and frames in Python, e.g. examples/phase_contrast.py:198-207);
this module is new.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import ops
from ._motion import lower
from .workloads import GAMMA, Block, Mesh, Trajectory

__all__ = ["Request", "Simulation", "Server", "latency_stats", "simulate_batch", "launch_iteration",
           "finish_iteration", "run_iteration", "SERVING_TUNING"]

# Work-unit shape used for every served request: a fixed node split keeps each
# request's reduction order independent of the batch it lands in.
SERVING_TUNING = ops.Tuning(split_nodes=16384, kz_cap=0)


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
    pod: object = None        # motion callable (lowered to the GPU when it can be)
    precision: str = "bf16x3"
    arrival: float = 0.0      # seconds after the start of the run
    weights: np.ndarray | None = None  # lumped mass weights; assembled on the device when None

    @property
    def n_nodes(self) -> int:
        return self.mesh.n_nodes

    @property
    def n_coils(self) -> int:
        return self.coils.shape[1]

    @property
    def work(self) -> float:
        """node*k-samples of the whole request."""
        return float(self.n_nodes) * self.traj.n_samples * self.frames


def footprint_bytes(req: Request) -> int:
    """Device bytes a request holds while admitted (state, inputs, outputs and
    its share of the batch workspace), estimated from its sizes."""
    N, S, C = req.n_nodes, req.traj.n_samples, req.n_coils
    E = req.mesh.elems.shape[0]
    state = N * (12 + 4 * 4 + 8 + 4 + 8 * C * 2)           # nodes, tissue, mass, Mxy/Mz, coils, Mxy columns
    traj = S * 16 + S * C * 8                              # k, t, one output frame
    mass_setup = E * 16 * 32 if req.weights is None else 0  # assembly triplets (transient)
    signal_ws = N * C * 8 + S * 64 + 16 * S * C * 8
    return int(state + traj + max(mass_setup, signal_ws) + (64 << 20))


def _upload_items(req: Request) -> list:
    """(host array, device dtype) of every input a Simulation uploads, in the
    order Simulation unpacks them."""
    t = req.traj
    items = [(req.mesh.nodes, torch.float32), (req.T1, torch.float32), (req.T2, torch.float32),
             (req.phi, torch.float32), (req.coils, torch.complex64), (t.kx, torch.float32),
             (t.ky, torch.float32), (t.kz, torch.float32), (t.t, torch.float32)]
    for b in req.blocks:
        items += [(b.rf, torch.complex64), (b.G, torch.float32), (b.dt, torch.float32)]
    if req.weights is not None:
        items.append((req.weights, torch.float32))
    return items


PINNED_KSPACE_MAX = 64 << 20  # bytes of a request's k-space frames kept in pinned memory


class Simulation:
    """Device-resident state of one request.  Construction queues the upload
    and the mass assembly on `stream` and records `ready` there.  `uploaded`:
    the request's inputs already on the device (in _upload_items order), when
    several requests were sent up together.  `pinned_kspace`: the k-space
    frames are allocated in pinned memory and copied there straight from the
    device (one-shot batches; a serving loop reuses pinned staging instead,
    which costs no new pinned allocation per request)."""

    def __init__(self, req: Request, device: torch.device, stream: torch.cuda.Stream | None = None,
                 uploaded: list | None = None, pinned_kspace: bool = False):
        from .Assemble import mass_lumped
        from .FiniteElements import FiniteElement, QuadratureRule
        self.req = req
        self.device = device
        self.stream = stream or torch.cuda.current_stream(device)
        self.frame = 0
        N, t = req.n_nodes, req.traj
        with torch.cuda.stream(self.stream):
            dev = uploaded if uploaded is not None else ops.upload_many(_upload_items(req), device)
            self.r0, self.T1, self.T2, self.phi, self.coils, kx, ky, kz, tt = dev[:9]
            self.blocks = [(dev[9 + 3 * i], dev[10 + 3 * i], dev[11 + 3 * i], b.t0, b.empty)
                           for i, b in enumerate(req.blocks)]
            if req.weights is not None:
                w = dev[-1]
            else:
                w = torch.from_numpy(np.ascontiguousarray(
                    mass_lumped(req.mesh.elems, req.mesh.nodes, FiniteElement(), QuadratureRule(order=2)),
                    np.float32)).to(device, non_blocking=True)
            idx = torch.arange(N + 1, dtype=torch.int32, device=device)
            self.M = ops.SparseCSC((N, N), idx, idx[:N], w)
            self.dB = torch.zeros(N, dtype=torch.float32, device=device)
            self.Mxy = torch.zeros(N, dtype=torch.complex64, device=device)
            self.Mz = torch.ones(N, dtype=torch.float32, device=device)
            self.readout = torch.empty(N, dtype=torch.complex64, device=device)
            self.cols = torch.empty((N, req.n_coils), dtype=torch.complex64, device=device)
            self.out = torch.empty((*t.shape, req.n_coils), dtype=torch.complex64, device=device)
            self.sig = ops.SignalInputs(M=self.M, kx=kx, ky=ky, kz=kz, t=tt, r0=self.r0, phi=self.phi, T2=self.T2,
                                        Mxy=self.cols)
            self.ready = torch.cuda.Event()
            self.ready.record(self.stream)
        # k-space frames land in pinned memory straight from the device when
        # asked (one-shot batches: no second host copy) and small enough,
        # else via pinned staging reused frame after frame
        shape = (req.frames, *t.shape, req.n_coils)
        if pinned_kspace and int(np.prod(shape)) * 8 <= PINNED_KSPACE_MAX:
            self._kspace_t = torch.empty(shape, dtype=torch.complex64, pin_memory=True)
            self.kspace = self._kspace_t.numpy()
        else:
            self._kspace_t = None
            self.kspace = np.empty(shape, np.complex64)

    @property
    def done(self) -> bool:
        return self.frame >= self.req.frames

    def enqueue_bloch(self, f: int) -> None:
        """Frame f's blocks on the current stream: the state is carried, Mxy
        spoiled after non-empty blocks (as BlochSolver does); the last
        block's final, unspoiled Mxy goes through every coil into the
        Signal's input columns."""
        req = self.req
        N = req.n_nodes
        src = None
        for bi, (rf, G, dt, t0, empty) in enumerate(self.blocks):
            last = bi == len(self.blocks) - 1
            if req.pod is not None:
                req.pod.update_timeshift(f * req.frame_ms + t0)
            inp = ops.BlochInputs(r0=self.r0, T1=self.T1, T2=self.T2, delta_B=self.dB, M0=1.0, gamma=GAMMA,
                                  rf=rf, G=G, dt=dt, Mxy0=self.Mxy, Mz0=self.Mz)
            final = self.Mxy if empty else (self.readout if last else None)
            ops.bloch_solve(inp, lower(req.pod, N, self.device), history=False, Mxy_final=final,
                            Mz_final=self.Mz, Mxy_carry=None if empty else self.Mxy, allocate_final=False)
            if last:
                src = self.Mxy if empty else self.readout
        ops.coil_expand(src, self.coils, out=self.cols)

    def motion(self, f: int):
        if self.req.pod is not None:
            self.req.pod.update_timeshift(f * self.req.frame_ms)
        return lower(self.req.pod, self.req.n_nodes, self.device)


BLOCH_STREAMS = 8  # helper streams over which a set of simulations' Bloch blocks is spread
_side_streams: dict = {}


def helper_streams(device: torch.device, k: int | None = None) -> list:
    """k helper streams of `device` (BLOCH_STREAMS when k is None), created
    once and reused."""
    k = BLOCH_STREAMS if k is None else k
    key = (device.index if device.index is not None else torch.cuda.current_device(), k)
    ss = _side_streams.get(key)
    if ss is None:
        ss = [torch.cuda.Stream(device=device) for _ in range(k)]
        _side_streams[key] = ss
    return ss


def enqueue_bloch_all(sims: list, frames: list | None = None) -> None:
    """Every simulation's Bloch blocks (frame frames[i], else its current
    frame) and coil columns.  The simulations are independent, so they are
    spread over helper streams forked from the current stream and joined back
    into it: small phantoms' sweeps run side by side instead of one after the
    other (in a captured graph: parallel branches)."""
    if not sims:
        return
    main = torch.cuda.current_stream(sims[0].device)
    k = min(BLOCH_STREAMS, len(sims))
    if k < 2:
        for i, s in enumerate(sims):
            s.enqueue_bloch(frames[i] if frames is not None else s.frame)
        return
    side = helper_streams(sims[0].device, BLOCH_STREAMS)[:k]
    fork = torch.cuda.Event()
    fork.record(main)
    for st in side:
        st.wait_event(fork)
    for i, s in enumerate(sims):
        with torch.cuda.stream(side[i % k]):
            s.enqueue_bloch(frames[i] if frames is not None else s.frame)
    for st in side:
        join = torch.cuda.Event()
        join.record(st)
        main.wait_event(join)


@dataclass
class Iteration:
    """One frame of a set of simulations, queued on a stream."""
    sims: list
    batch: object
    host: list
    stream: torch.cuda.Stream
    keep: list


def launch_iteration(sims: list[Simulation], tuning: ops.Tuning = SERVING_TUNING) -> Iteration:
    """Queues one frame of every simulation on the current stream: their
    Bloch blocks, one persistent launch for all split-BF16 Signals (float32
    requests run their own CUDA-core Signal), then copies of the outputs to
    pinned host buffers.  Does not wait; finish_iteration() does."""
    stream = torch.cuda.current_stream(sims[0].device)
    for s in sims:
        stream.wait_event(s.ready)
    enqueue_bloch_all(sims)
    batch, keep = [], []
    for s in sims:
        mo = s.motion(s.frame)
        keep.append(mo)
        if s.req.precision == "bf16x3":
            batch.append((s.sig, mo, s.out))
        else:
            ops.signal(s.sig, mo, s.req.precision, out=s.out, sync=False)
    sb = ops.SignalBatch(batch, tuning) if batch else None
    if sb is not None:
        sb.enqueue()
    host = []
    for s in sims:
        if s._kspace_t is not None:
            s._kspace_t[s.frame].copy_(s.out, non_blocking=True)
            host.append(None)
        else:
            h = torch.empty(s.out.shape, dtype=torch.complex64, pin_memory=True)
            h.copy_(s.out, non_blocking=True)
            host.append(h)
    return Iteration(sims, sb, host, stream, keep)


def finish_iteration(it: Iteration) -> None:
    """Waits for a launched iteration, raises the errors its device work
    found, and files each simulation's frame."""
    if it.batch is not None:
        it.batch.status()
    it.stream.synchronize()
    for s, h in zip(it.sims, it.host):
        if h is not None:
            s.kspace[s.frame] = h.numpy()
        s.frame += 1


def run_iteration(sims: list[Simulation], tuning: ops.Tuning = SERVING_TUNING) -> None:
    """launch_iteration + finish_iteration."""
    if sims:
        finish_iteration(launch_iteration(sims, tuning))


_copy_streams: dict = {}


def _copy_stream(device: torch.device) -> torch.cuda.Stream:
    key = device.index if device.index is not None else torch.cuda.current_device()
    st = _copy_streams.get(key)
    if st is None:
        st = torch.cuda.Stream(device=device)
        _copy_streams[key] = st
    return st


def _split_by_work(requests: list[Request], parts: int) -> list[list[Request]]:
    """Consecutive groups of requests with about equal node*k-sample work."""
    total = sum(r.work for r in requests)
    groups, cur, acc = [], [], 0.0
    for r in requests:
        cur.append(r)
        acc += r.work
        if len(groups) < parts - 1 and acc >= total * (len(groups) + 1) / parts:
            groups.append(cur)
            cur = []
    if cur:
        groups.append(cur)
    return groups


def simulate_batch(requests: list[Request], device: torch.device | None = None,
                   tuning: ops.Tuning | None = None, parts: int = 4) -> list[np.ndarray]:
    """One frame of many simulations, host arrays in and host arrays out.

    The requests go in `parts` consecutive groups of about equal work.  Each
    group's inputs go up through pinned staging in one pass (copies on
    several threads) and one host-to-device transfer.  Its Bloch blocks and
    coil expansions run, then one persistent tensor-core launch contracts all
    of its Signals, and the k-spaces come back through pinned memory.  The
    host stages the next group while the device works on the last one, and
    its transfer (on a copy stream) overlaps that work.  A request's result
    does not depend on its group.  Returns one (n_ro,
    n_lines, n_kz, C) complex64 array per request."""
    device = device or ops.require_cuda()
    stream = torch.cuda.current_stream(device)
    # uploads go through a copy stream: a group's transfer overlaps the
    # previous group's launch, and the launch stream waits for it
    copy = _copy_stream(device)
    launched = []
    for group in _split_by_work(requests, max(1, parts)):
        items, counts = [], []
        for r in group:
            it = _upload_items(r)
            items += it
            counts.append(len(it))
        dev = []
        if items:
            with torch.cuda.stream(copy):
                dev = ops.upload_many(items, device)
            ready = torch.cuda.Event()
            ready.record(copy)
            stream.wait_event(ready)
            dev[0].record_stream(stream)  # the views share one allocation
        sims, k = [], 0
        for r, c in zip(group, counts):
            sims.append(Simulation(r, device, stream, uploaded=dev[k:k + c], pinned_kspace=True))
            k += c
        launched.append((sims, launch_iteration(sims, tuning or SERVING_TUNING)))
    out = []
    for sims, it in launched:
        finish_iteration(it)
        out += [s.kspace[0] for s in sims]
    return out


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
    iterations: int = 0        # launches the request took part in
    peers_max: int = 0         # most other requests in one of its launches


@dataclass
class Server:
    """Continuous-batching request loop on one GPU.

    slots:       requests that may be in flight at the same time;
    hbm_budget:  bytes of device memory the admitted requests may hold
                 (0: 80% of the free memory at start)."""
    device: torch.device = None
    slots: int = 16
    hbm_budget: int = 0
    tuning: ops.Tuning = SERVING_TUNING
    results: list = field(default_factory=list)

    def __post_init__(self):
        self.device = self.device or ops.require_cuda()
        if not self.hbm_budget:
            free, _ = torch.cuda.mem_get_info(self.device)
            self.hbm_budget = int(free * 0.8)
        self._side = torch.cuda.Stream(device=self.device)
        self._main = torch.cuda.Stream(device=self.device)

    def serve(self, requests: list[Request], realtime: bool = True) -> list[Served]:
        """Runs the requests, each arriving at req.arrival seconds after the
        start (when realtime; otherwise all at once) and admitted when a slot
        and memory allow; returns one record per request with its times and
        k-space.  A request that fails at set-up or in a launch is reported
        with its error; the others go on."""
        torch.cuda.set_device(self.device)
        order = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        items = [Served(r, r.arrival if realtime else 0.0) for r in order]
        pending = list(items)
        active: list[tuple[Served, Simulation, int]] = []
        in_use = 0

        def now():
            return time.perf_counter() - t0

        def admit():
            nonlocal in_use
            while pending and (not realtime or pending[0].arrival <= now()):
                need = footprint_bytes(pending[0].req)
                if len(active) + len(joining) >= self.slots or \
                        ((active or joining) and in_use + need > self.hbm_budget):
                    return
                item = pending.pop(0)
                item.admitted = now()
                try:
                    with torch.cuda.stream(self._side):
                        sim = Simulation(item.req, self.device, self._side)
                except Exception as exc:  # noqa: BLE001 - the request fails, the server goes on
                    item.error = f"{type(exc).__name__}: {exc}"
                    item.finished = now()
                    continue
                joining.append((item, sim, need))
                in_use += need

        joining: list = []
        while pending or active or joining:
            active += joining
            joining = []
            if not active:
                admit()
                if not joining and pending and realtime:
                    time.sleep(max(0.0, min(pending[0].arrival - now(), 0.01)))
                continue
            try:
                with torch.cuda.stream(self._main):
                    it = launch_iteration([s for _, s, _ in active], self.tuning)
                # requests arriving meanwhile are set up while the launch runs
                admit()
                finish_iteration(it)
            except Exception as exc:  # noqa: BLE001 - fail the launch's requests, keep serving
                for item, _, need in active:
                    item.error = f"{type(exc).__name__}: {exc}"
                    item.finished = now()
                    in_use -= need
                active = []
                continue
            t_done = now()
            keep = []
            for item, sim, need in active:
                item.iterations += 1
                item.peers_max = max(item.peers_max, len(active) - 1)
                if sim.done:
                    item.kspace = sim.kspace
                    item.finished = t_done
                    in_use -= need
                else:
                    keep.append((item, sim, need))
            active = keep
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
                    "throughput_node_samples_per_s": work / span if span > 0 else None, "span_s": span,
                    "max_requests_per_launch": 1 + max((it.peers_max for it in done), default=0)})
        return out
