"""Benchmark of the simulation hot path on one node.

Workload (phase-contrast flow, the metric's configuration): a 200k-node P1
tube (radius 12 mm, length 100 mm) with Poiseuille flow (peak 1 m/s) moving
the nodes as a rank-1 PODVelocity, off-resonance ~N(0, 20 Hz), T1 ~ U[0.8,
1.2] s, T2 ~ U[50, 100] ms, lumped P1 mass weights, a 3-D Cartesian
96 x 96 x 32 readout (FOV 0.1 m, sample time set by the readout index, so 96
distinct times) and 4 velocity encodings (reference + 3 axes, VENC 1.5 m/s).

One step simulates one cardiac frame: the fused Bloch sweep of the
phase-contrast imaging block for the 4 encodings (final-state form, motion on
the GPU), then the mass-weighted NUDFT of the 4 encodings at once
(V = 4 columns).  Units: node*k-sample = nodes x k-space samples per step.
Each rank simulates its own frame (frames are independent): weak scaling, no
collective on the data path.  Inputs are synthetic and seeded.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision bf16x3|f32]
  python bench.py --impl reference ...   (CPU restatement of the reference)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "node*k-sample/s"
N_NODES = 200_000
RES = (96, 96, 32)
FOV = (0.1, 0.1, 0.1)
RADIUS, LENGTH = 0.012, 0.1
VENC = 1.5


def build_case(seed: int = 0, n_nodes: int = N_NODES):
    """Host-side synthetic inputs (numpy)."""
    from feelmri_b200 import workloads as W
    mesh = W.tube(n_nodes, RADIUS, LENGTH)
    N = mesh.n_nodes
    T1, T2 = W.tissue(N, seed)
    phi = W.off_resonance(N, 20.0, seed + 1)
    traj = W.cartesian(res=RES, fov=FOV)
    vel = W.poiseuille_velocity(mesh.nodes, RADIUS, v_max=1.0, period=1000.0, n_frames=20)
    blocks = [W.pc_imaging_block(0.0, enc, venc=VENC) for enc in W.PC_ENCODINGS]
    return dict(mesh=mesh, N=N, T1=T1, T2=T2, phi=phi, traj=traj, vel=vel, blocks=blocks,
                dB=np.zeros(N, np.float32))


# --------------------------------------------------------------- clocks --

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, period_ms: int = 50):
        self.idx = device_index
        self.period_ms = period_ms
        self.proc = None
        self.lines: list[str] = []
        self._first = threading.Event()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region starts once samples flow
            self._first.wait(timeout=10.0)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self._first.set()

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- GPU arm --

def run_gpu(args) -> dict | None:
    import torch
    import scipy.sparse as sp
    from feelmri_b200 import _lib, ops
    from feelmri_b200._motion import lower
    from feelmri_b200.Assemble import mass_lumped
    from feelmri_b200.Bloch import BlochSolver
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    from feelmri_b200.MRI import Signal
    from feelmri_b200 import workloads as W

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    case = build_case(n_nodes=args.nodes)
    N = case["N"]
    traj = case["traj"]
    S = traj.n_samples
    V = len(W.PC_ENCODINGS)
    vel = case["vel"]
    frame_ms = 40.0
    vel.update_timeshift(frame_ms * rank)

    # one-time setup (untimed, as the reference assembles the mass "just once")
    fe, qr = FiniteElement(), QuadratureRule(order=2)
    w = mass_lumped(case["mesh"].elems, case["mesh"].nodes, fe, qr)
    up = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)  # noqa
    r0 = up(case["mesh"].nodes.astype(np.float32))
    T1, T2, dB = up(case["T1"]), up(case["T2"]), up(case["dB"])
    blocks = []
    for b in case["blocks"]:
        blocks.append((up(b.rf, torch.complex64), up(b.G), up(b.dt.astype(np.float32)), b.t0))
    Minds = ops.SparseCSC((N, N), up(np.arange(N + 1, dtype=np.int32), torch.int32),
                          up(np.arange(N, dtype=np.int32), torch.int32), up(w.astype(np.float32)))
    sig_in = ops.SignalInputs(M=Minds, kx=up(traj.kx), ky=up(traj.ky), kz=up(traj.kz), t=up(traj.t), r0=r0,
                              phi=up(case["phi"]), T2=T2, Mxy=torch.empty((N, V), dtype=torch.complex64, device=dev))
    Mz_tmp = torch.empty((N,), dtype=torch.float32, device=dev)
    zero_m = torch.zeros((N,), dtype=torch.complex64, device=dev)
    one_z = torch.ones((N,), dtype=torch.float32, device=dev)
    out = torch.empty((*traj.shape, V), dtype=torch.complex64, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    precision = args.precision

    def step():
        for e, (rf, G, dt, t0) in enumerate(blocks):
            vel.update_timeshift(frame_ms * rank + t0)
            motion = lower(vel, N, dev)
            inp = ops.BlochInputs(r0=r0, T1=T1, T2=T2, delta_B=dB, M0=1.0, gamma=W.GAMMA, rf=rf, G=G, dt=dt,
                                  Mxy0=zero_m, Mz0=one_z)
            # each encoding's final transverse magnetisation lands in column e
            ops.bloch_solve(inp, motion, history=False, Mxy_final=sig_in.Mxy[:, e], Mz_final=Mz_tmp)
        vel.update_timeshift(frame_ms * rank)
        return ops.signal(sig_in, lower(vel, N, dev), precision, out=out)

    stream = torch.cuda.current_stream(dev)
    ctx = ops.ctx_for(dev)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    _lib.timing_reset(ctx)
    _lib.timing(ctx, True)
    launches0 = _lib.launch_count()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize(dev)
        for i in range(args.steps):
            flush.zero_()  # L2 (126 MB) flushed between timed steps, outside the events
            starts[i].record(stream)
            step()
            ends[i].record(stream)
        torch.cuda.synchronize(dev)
    launches = _lib.launch_count() - launches0
    _lib.timing(ctx, False)
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    kname = "signal_tc" if precision == "bf16x3" else "signal_f32"
    k_ms, k_n = _lib.timing_query(ctx, kname)
    b_ms, b_n = _lib.timing_query(ctx, "bloch")
    if dist:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())

    # correctness spot check of this run's output against FP64 (a few samples)
    from oracle import fp64
    Mxy_host = sig_in.Mxy.cpu().numpy()
    idx = np.random.default_rng(0).choice(S, 256, replace=False)
    disp = None
    M_host = sp.diags(w).tocsc()
    calls = np.unique(traj.t.reshape(-1)[idx])
    from feelmri_b200.MRI import signal_call_times
    run_times = signal_call_times(traj.t)[1:]
    disp = np.stack([vel(float(t)) for t in run_times])
    ref = fp64.signal(M_host, traj.kx, traj.ky, traj.kz, traj.t, case["mesh"].nodes.astype(np.float32),
                      case["phi"], case["T2"], Mxy_host, disp=disp, pi_mode="float", sample_idx=idx)
    got = out.cpu().numpy().reshape(S, V)[idx]
    rel = fp64.rel_l2(got, ref)

    # Bloch sweep in its API-exact history form (HBM-bound: every node-step
    # writes c64 Mxy + f32 Mz): one encoding block, timed alone, untimed by
    # the step.  Algorithmic bytes = N n_t 12 written + N 36 read (position,
    # T1, T2, dB, initial state) + n_t 24 (rf, G, dt) + the rank-1 modes.
    rf, G, dt, t0 = blocks[1]
    vel.update_timeshift(frame_ms * rank + t0)
    hist_motion = lower(vel, N, dev)
    hinp = ops.BlochInputs(r0=r0, T1=T1, T2=T2, delta_B=dB, M0=1.0, gamma=W.GAMMA, rf=rf, G=G, dt=dt,
                           Mxy0=zero_m, Mz0=one_z)
    ops.bloch_solve(hinp, hist_motion, history=True)
    torch.cuda.synchronize(dev)
    h_ms = []
    for _ in range(5):
        flush.zero_()
        a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a_ev.record(stream)
        ops.bloch_solve(hinp, hist_motion, history=True)
        b_ev.record(stream)
        b_ev.synchronize()
        h_ms.append(a_ev.elapsed_time(b_ev))
    n_t = int(rf.shape[0])
    h_bytes = float(N) * n_t * 12 + float(N) * (12 + 12 + 12 + 12) + n_t * 24
    bloch_hist = {"bound": "hbm", "ms": statistics.median(h_ms), "bytes": h_bytes,
                  "achieved": h_bytes / (statistics.median(h_ms) / 1e3) / 1e9, "unit": "GB/s",
                  "node_steps_per_s": float(N) * n_t / (statistics.median(h_ms) / 1e3), "n_t": n_t}

    result = None
    if rank == 0:
        units = float(N) * S * world
        value = units / (total_ms / args.steps / 1e3)
        # roofline of the dominant kernel
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() \
            else {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "note": "fallback"}
        k_avg_s = (k_ms / max(k_n, 1)) / 1e3
        if precision == "bf16x3":
            flops = 3 * 8.0 * V * float(N) * S  # issued split-BF16 MMA flops per launch
            roof = {"bound": "tensor", "achieved": flops / k_avg_s / 1e12, "peak": peaks["bf16_tflops"],
                    "unit": "TFLOP/s"}
        else:
            flops = (8.0 + 8.0 * V) * float(N) * S  # algorithmic FP32 flops per launch (phase + complex MACs)
            roof = {"bound": "tensor", "achieved": flops / k_avg_s / 1e12, "peak": peaks["bf16_tflops"],
                    "unit": "TFLOP/s"}
        roof["frac"] = roof["achieved"] / roof["peak"]
        # DRAM bytes of one full-size launch of the dominant kernel, from one ncu
        # capture (dram__bytes_read.sum + dram__bytes_write.sum, a one-pass metric
        # pair) of this command: 16.96 MB read + 0.14 MB written (16.7-17.1 MB over
        # captures).  The node data is read from DRAM about once and reused from L2
        # by the work units.
        roof["traffic"] = 17.10e6 if precision == "bf16x3" and N == 200740 else None
        roof["traffic_unit"] = "bytes per launch"
        roof["kernel"] = kname
        roof["kernel_ms"] = k_ms / max(k_n, 1)
        roof["peak_source"] = "measured" if "note" not in peaks else "fallback"
        result = {
            "metric": METRIC, "value": value, "unit": "node*k-sample/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3" if precision == "bf16x3" else "f32",
            "data": "synthetic (seeded mesh, tissue, flow and trajectory)",
            "config": {"workload": f"phase-contrast flow: {N // 1000}k-node P1 tube, Poiseuille 1 m/s, "
                                   "96x96x32 Cartesian, 4 velocity encodings (VENC 1.5 m/s), off-resonance N(0,20 Hz)",
                       "nodes": N, "k_samples": S, "columns": V, "distinct_times": 96,
                       "precision": precision, "l2": "flushed (512 MB write) between timed steps",
                       "parallelism": f"frames x{world}" if world > 1 else "single GPU"},
            "rel_l2_vs_fp64": rel,
            "roofline": roof,
            "bloch_ms_per_step": b_ms / args.steps,
            "bloch_history_roofline": dict(bloch_hist, peak=peaks["hbm_gbs"],
                                           frac=bloch_hist["achieved"] / peaks["hbm_gbs"]),
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
        if args.e2e:
            result["e2e"] = run_e2e(args, case, w, precision)
        if args.cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(case, w, budget_s=args.cpu_seconds)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def run_e2e(args, case, w, precision) -> dict:
    """Same step through the public API with host (numpy) buffers: the
    sequence driver for the 4 encodings, then MRI.Signal."""
    import scipy.sparse as sp
    import torch
    from feelmri_b200.Bloch import BlochSolver
    from feelmri_b200.MRI import Signal
    from feelmri_b200 import workloads as W
    N = case["N"]
    traj = case["traj"]
    M = sp.lil_matrix((N, N), dtype=np.float64)
    M.setdiag(w)
    nodes32 = case["mesh"].nodes.astype(np.float32)

    def step():
        cols = []
        for b in case["blocks"]:
            s = BlochSolver([b], nodes32, M0=1.0, T1=case["T1"], T2=case["T2"], delta_B=case["dB"],
                            gamma=W.GAMMA, pod_trajectory=case["vel"])
            m, _ = s.solve()
            cols.append(m[:, 0])
        Mxy = np.stack(cols, axis=1)
        case["vel"].update_timeshift(0.0)
        K = Signal(0, M, traj.points, traj.t, nodes32, case["phi"], case["T2"], Mxy, case["vel"],
                   precision=precision if precision == "bf16x3" else None)
        return K

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    n = max(5, min(args.steps, 20))
    t0 = time.perf_counter()
    for _ in range(n):
        K = step()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / n
    V = K.shape[-1]
    n_blocks = len(case["blocks"])
    # per solver: nodes, T1, T2, delta_B (initial state is filled on the device);
    # per block: rf, G, dt.  Signal: M (indptr, indices, data), k-space and
    # times, nodes, phi, T2 and the Mxy columns.
    h2d = (n_blocks * (nodes32.nbytes + 3 * N * 4)
           + sum(b.rf.nbytes + b.G.nbytes + b.dt.astype(np.float32).nbytes for b in case["blocks"])
           + (N + 1) * 4 + N * 4 + N * 4 + sum(p.nbytes for p in traj.points) + traj.t.nbytes
           + nodes32.nbytes + 2 * N * 4 + N * V * 8)
    d2h = K.nbytes + n_blocks * N * (8 + 4)
    return {"value": float(N) * traj.n_samples / dt, "unit": "node*k-sample/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "timer": "host wall clock around the public calls, device synchronised"}


# -------------------------------------------------------- CPU baseline --

def _host_motion(motion, t: float) -> np.ndarray:
    """A POD / PODVelocity / PODSum callable evaluated on the host only: the
    weights as the class computes them (spline at the folded time, times t for
    velocities, Motion.py:240-290) and the modes x weights product by the
    oracle's restatement of POD.cpp, so the CPU baseline runs no device code."""
    import oracle
    from feelmri_b200.Motion import PODSum, PODVelocity
    if isinstance(motion, PODSum):
        return _host_motion(motion.pod1, t) + _host_motion(motion.pod2, t)
    motion._evaluate_weights(motion._fold_time(t + motion.timeshift))
    if isinstance(motion, PODVelocity):
        motion._weights *= t
    return oracle.tensordot(motion._modes, motion._weights)


def cpu_baseline(case, w, budget_s: float = 15.0, threads: int | None = None) -> dict:
    """The C restatement of the reference's Signal (reference compiler flags,
    one thread per core over node ranges, partial k-spaces summed as
    gather_data does) on a bounded sample: all nodes x a subset of readout
    indices, sized to a few seconds of CPU work, scaled to node*k-samples/s."""
    import oracle
    import scipy.sparse as sp
    traj = case["traj"]
    N = case["N"]
    threads = threads or max(1, os.cpu_count() or 1)
    M = sp.diags(w.astype(np.float32)).tocsc()
    Mxy = (np.ones((N, 4)) * (0.1 + 0.05j)).astype(np.complex64)
    nodes32 = case["mesh"].nodes.astype(np.float32)
    n_ro = 1
    while True:
        sl = slice(0, n_ro)
        kx, ky, kz, t = (a[sl] for a in (*traj.points, traj.t))
        disp = np.stack([_host_motion(case["vel"], float(tt)) for tt in np.unique(t)])
        t0 = time.perf_counter()
        oracle.signal(M, kx, ky, kz, t, nodes32, case["phi"], case["T2"], Mxy, disp=disp, dtype=np.float32,
                      threads=threads, flavour="fast")
        el = time.perf_counter() - t0
        if el > budget_s / 4 or n_ro >= traj.shape[0]:
            break
        n_ro = min(traj.shape[0], max(n_ro * 2, int(n_ro * budget_s / 4 / max(el, 1e-3))))
    samples = int(np.prod(kx.shape))
    return {"value": float(N) * samples / el, "unit": "node*k-sample/s", "cores": threads, "kind": "port",
            "sample": f"all {N} nodes x {samples} k-samples ({n_ro} readout indices of 96), 4 columns, "
                      f"Signal only, {el:.1f} s"}


def run_reference(args) -> dict | None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    case = build_case()
    from feelmri_b200 import workloads as W
    from oracle import fp64
    w = fp64.lumped_p1(case["mesh"].elems, case["mesh"].nodes)
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(case, w, budget_s=4.0)
    for _ in range(args.steps):
        vals.append(cpu_baseline(case, w, budget_s=max(4.0, args.cpu_seconds / max(args.steps, 1))))
    v = statistics.median(x["value"] for x in vals)
    cb = dict(vals[-1])
    cb["value"] = v
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "node*k-sample/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(case["N"]) * case["traj"].n_samples / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded mesh, tissue, flow and trajectory)",
            "config": {"workload": "phase-contrast flow: 200k-node P1 tube, Poiseuille 1 m/s, 96x96x32 Cartesian, "
                                   "4 velocity encodings (VENC 1.5 m/s), off-resonance N(0,20 Hz)",
                       "implementation": "CPU restatement of the reference's Signal (the reference's native "
                                         "modules cannot be built here: Eigen is fetched from the network)"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "node*k-sample/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ------------------------------------------------------- batching (cfg 3) --

BATCH_PHANTOMS = 64


def build_batch_case(n_phantoms: int = BATCH_PHANTOMS, seed: int = 4):
    """Phantoms of uneven size: node counts log-uniform in [5k, 300k], shapes
    cycling cylinder / ellipsoid / tube; SPAMM tagging (8 mm) then a 15-degree
    GRE excitation; per phantom a 3-D Cartesian grid or a stack of spirals of
    4k-200k samples (log-uniform) and 1 or 2 receive coils."""
    from feelmri_b200 import workloads as W
    rng = np.random.default_rng(seed)
    shapes = (W.cylinder, W.ellipsoid, W.tube)
    out = []
    for i in range(n_phantoms):
        n = int(np.exp(rng.uniform(np.log(5e3), np.log(3e5))))
        mesh = shapes[i % 3](n)
        N = mesh.n_nodes
        T1, T2 = W.tissue(N, seed + i)
        s_target = np.exp(rng.uniform(np.log(4e3), np.log(2e5)))
        n_kz = int(rng.choice([8, 16, 32]))
        if i % 2 == 0:
            side = max(4, int(round(np.sqrt(s_target / n_kz))))
            traj = W.cartesian(res=(side, side, n_kz))
        else:
            il = int(rng.choice([8, 16, 32]))
            n_ro = max(16, int(round(s_target / (il * n_kz))))
            traj = W.spiral_stack(n_ro=n_ro, n_interleaves=il, n_kz=n_kz)
        coils = W.coil_maps(mesh.nodes, int(rng.integers(1, 3)), seed=seed + i)
        blocks = [W.spamm_block(0.0), W.hard_pulse_block(3.0, 15.0, 5.0)]
        out.append(dict(mesh=mesh, N=N, T1=T1, T2=T2, phi=W.off_resonance(N, 20.0, seed + i), traj=traj,
                        coils=coils, blocks=blocks))
    return out


def run_batching(args) -> dict:
    """One step = one frame of every phantom: Bloch (SPAMM block, then the GRE
    block; final states only), coil columns, then the mass-weighted NUDFT of
    all phantoms.  Split-BF16 form: one persistent tensor-core launch with
    autotuned units; FP32 form: one CUDA-core Signal per phantom.  Each form's
    step is captured in a CUDA graph and replayed."""
    import torch
    import scipy.sparse as sp
    from feelmri_b200 import ops, autotune
    from feelmri_b200._motion import lower
    from feelmri_b200.Assemble import mass_lumped
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    from feelmri_b200 import workloads as W
    from oracle import fp64

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    case = build_batch_case(args.phantoms)
    build_s = time.perf_counter() - t0
    up = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)  # noqa
    fe, qr = FiniteElement(), QuadratureRule(order=2)
    ph = []
    for c in case:
        N = c["N"]
        w = mass_lumped(c["mesh"].elems, c["mesh"].nodes, fe, qr)
        V = c["coils"].shape[1]
        d = dict(N=N, V=V, S=c["traj"].n_samples, w=w)
        d["r0"] = up(c["mesh"].nodes.astype(np.float32))
        d["T1"], d["T2"] = up(c["T1"]), up(c["T2"])
        d["dB"] = torch.zeros(N, dtype=torch.float32, device=dev)
        d["phi"] = up(c["phi"])
        d["coils"] = up(c["coils"], torch.complex64)
        d["blocks"] = [(up(b.rf, torch.complex64), up(b.G), up(b.dt.astype(np.float32))) for b in c["blocks"]]
        d["Mxy"] = torch.zeros(N, dtype=torch.complex64, device=dev)
        d["Mz"] = torch.ones(N, dtype=torch.float32, device=dev)
        d["zero"] = torch.zeros(N, dtype=torch.complex64, device=dev)
        d["one"] = torch.ones(N, dtype=torch.float32, device=dev)
        d["read"] = torch.empty(N, dtype=torch.complex64, device=dev)
        d["cols"] = torch.empty((N, V), dtype=torch.complex64, device=dev)
        t = c["traj"]
        M = ops.SparseCSC((N, N), up(np.arange(N + 1, dtype=np.int32), torch.int32),
                          up(np.arange(N, dtype=np.int32), torch.int32), up(w.astype(np.float32)))
        d["sig"] = ops.SignalInputs(M=M, kx=up(t.kx), ky=up(t.ky), kz=up(t.kz), t=up(t.t), r0=d["r0"], phi=d["phi"],
                                    T2=d["T2"], Mxy=d["cols"])
        d["motion"] = lower(None, N, dev)
        d["out_tc"] = torch.empty((*t.shape, V), dtype=torch.complex64, device=dev)
        d["out_32"] = torch.empty((*t.shape, V), dtype=torch.complex64, device=dev)
        ph.append(d)
    units = float(sum(d["N"] * d["S"] for d in ph))

    def bloch_all():
        for d in ph:
            (rf0, G0, dt0), (rf1, G1, dt1) = d["blocks"]
            inp = ops.BlochInputs(r0=d["r0"], T1=d["T1"], T2=d["T2"], delta_B=d["dB"], M0=1.0, gamma=W.GAMMA,
                                  rf=rf0, G=G0, dt=dt0, Mxy0=d["zero"], Mz0=d["one"])
            # SPAMM: Mz carried, Mxy spoiled (BlochSolver zeroes it after a non-empty block)
            ops.bloch_solve(inp, d["motion"], history=False, Mxy_final=d["Mxy"], Mz_final=d["Mz"])
            inp = ops.BlochInputs(r0=d["r0"], T1=d["T1"], T2=d["T2"], delta_B=d["dB"], M0=1.0, gamma=W.GAMMA,
                                  rf=rf1, G=G1, dt=dt1, Mxy0=d["zero"], Mz0=d["Mz"])
            ops.bloch_solve(inp, d["motion"], history=False, Mxy_final=d["read"], Mz_final=d["Mz"])
            ops.coil_expand(d["read"], d["coils"], out=d["cols"])

    # autotuned units for this batch (timed on the batch itself)
    problems = [(d["sig"], d["motion"], d["out_tc"]) for d in ph]
    bloch_all()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tuning, tried = autotune.tune(problems, force=True)
    tune_s = time.perf_counter() - t0
    batch = ops.SignalBatch(problems, tuning)

    def step_tc():
        bloch_all()
        batch.enqueue()

    def step_32():
        bloch_all()
        for d in ph:
            ops.signal(d["sig"], d["motion"], "f32", out=d["out_32"], sync=False)

    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    res = {}
    for name, fn in (("bf16x3", step_tc), ("f32", step_32)):
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 1)):
                fn()
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            fn()
        launches0 = _lib_launches()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with torch.cuda.stream(stream):
            g.replay()  # one untimed replay
            for a, b in ev:
                flush.zero_()
                a.record(stream)
                g.replay()
                b.record(stream)
        stream.synchronize()
        ms = [a.elapsed_time(b) for a, b in ev]
        res[name] = {"ms_per_step": statistics.median(ms), "value": units / (statistics.median(ms) / 1e3)}
        del g
    batch.status()
    # spot check of the split-BF16 result of the largest and smallest phantom against FP64
    errs = []
    for i in (int(np.argmax([d["N"] for d in ph])), int(np.argmin([d["N"] for d in ph]))):
        d = ph[i]
        S = d["S"]
        idx = np.random.default_rng(i).choice(S, min(S, 128), replace=False)
        t = case[i]["traj"]
        ref = fp64.signal(sp.diags(d["w"]).tocsc(), t.kx, t.ky, t.kz, t.t, case[i]["mesh"].nodes.astype(np.float32),
                          case[i]["phi"], case[i]["T2"], d["cols"].cpu().numpy(), pi_mode="float", sample_idx=idx)
        errs.append(fp64.rel_l2(d["out_tc"].cpu().numpy().reshape(S, -1)[idx], ref))
        errs.append(fp64.rel_l2(d["out_32"].cpu().numpy().reshape(S, -1)[idx], ref))
    tc, f32 = res["bf16x3"], res["f32"]
    return {
        "metric": METRIC, "value": tc["value"], "unit": "node*k-sample/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tc["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic (seeded phantoms, sequences and trajectories)",
        "config": {"workload": f"batching: {len(ph)} phantoms, nodes log-uniform 5k-300k "
                               f"(total {sum(d['N'] for d in ph)}), SPAMM (8 mm) + 15-degree GRE, Cartesian or "
                               f"stack-of-spirals 4k-200k samples, 1-2 coils",
                   "node_samples_per_step": units, "precision": "bf16x3 (one persistent launch) vs f32 "
                   "(one launch per phantom)", "l2": "flushed (512 MB write) between timed replays",
                   "graph": "each step captured once in a CUDA graph and replayed"},
        "f32": {"value": f32["value"], "ms_per_step": f32["ms_per_step"]},
        "speedup_vs_f32": f32["ms_per_step"] / tc["ms_per_step"],
        "rel_l2_vs_fp64": {"bf16x3_max": max(errs[0::2]), "f32_max": max(errs[1::2])},
        "tuning": {"split_nodes": tuning.split_nodes, "kz_cap": tuning.kz_cap, "search_s": tune_s,
                   "tried_ms": {f"{k.split_nodes}/{k.kz_cap}": v for k, v in tried.items()}},
        "setup_s": {"phantoms": build_s},
    }


# ------------------------------------------------------ precision (cfg 2) --

def run_precision(args) -> dict:
    """Ellipsoid phantom (semi-axes 60/50/40 mm), POD motion (rank 10,
    Phi ~ N(0, 1 mm), sinusoidal weights, 800 ms cycle), 3-D radial readout
    (256 readout points x 4096 spokes, |k| <= 500 1/m, one distinct time per
    readout point), 8 Gaussian receive coils; one frame per step (a
    15-degree excitation, then the Signal of all coils).  Split-BF16 and FP32
    forms, each against the FP64 oracle on a seeded subset of samples."""
    import torch
    import scipy.sparse as sp
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    from feelmri_b200.Assemble import mass_lumped
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    from feelmri_b200.MRI import signal_call_times
    from feelmri_b200 import workloads as W
    from oracle import fp64

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    mesh = W.ellipsoid(args.nodes if args.nodes != N_NODES else 500_000)
    N = mesh.n_nodes
    traj = W.radial3d(n_ro=256, n_spokes=args.spokes, kmax=500.0)
    S = traj.n_samples
    C = 8
    T1, T2 = W.tissue(N, 2)
    phi = W.off_resonance(N, 20.0, 2)
    coils = W.coil_maps(mesh.nodes, C, seed=3)
    pod = W.sinusoidal_pod(N, n_modes=10, amp=1e-3, period=800.0, n_frames=20, seed=2)
    w = mass_lumped(mesh.elems, mesh.nodes, FiniteElement(), QuadratureRule(order=2))
    up = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)  # noqa
    r0 = up(mesh.nodes.astype(np.float32))
    M = ops.SparseCSC((N, N), up(np.arange(N + 1, dtype=np.int32), torch.int32),
                      up(np.arange(N, dtype=np.int32), torch.int32), up(w.astype(np.float32)))
    # magnetisation after a 15-degree excitation, through every coil
    m0 = np.full(N, np.sin(np.deg2rad(15.0)), np.complex64)
    cols = up(m0[:, None] * coils, torch.complex64)
    sig = ops.SignalInputs(M=M, kx=up(traj.kx), ky=up(traj.ky), kz=up(traj.kz), t=up(traj.t), r0=r0, phi=up(phi),
                           T2=up(T2), Mxy=cols)
    res = {}
    outs = {}
    for prec in ("bf16x3", "f32"):
        out = torch.empty((*traj.shape, C), dtype=torch.complex64, device=dev)
        ms = []
        for f in range(args.warmup + args.steps):
            pod.update_timeshift(40.0 * f)
            mo = lower(pod, N, dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            ops.signal(sig, mo, prec, out=out)
            b.record()
            b.synchronize()
            if f >= args.warmup:
                ms.append(a.elapsed_time(b))
        res[prec] = statistics.median(ms)
        outs[prec] = out.cpu().numpy().reshape(S, C)
    # FP64 oracle on a seeded subset of the last frame's samples
    idx = np.random.default_rng(2).choice(S, args.check_samples, replace=False)
    times = signal_call_times(traj.t)[1:]

    class _RunDisp:  # displacement of run g, computed only for the runs the subset touches
        def __getitem__(self, g):
            return pod(float(times[g]))

    disp = _RunDisp()
    ref = fp64.signal(sp.diags(w).tocsc(), traj.kx, traj.ky, traj.kz, traj.t, mesh.nodes.astype(np.float32), phi, T2,
                      cols.cpu().numpy(), disp=disp, pi_mode="float", sample_idx=idx)
    units = float(N) * S
    return {
        "metric": METRIC, "value": units / (res["bf16x3"] / 1e3), "unit": "node*k-sample/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["bf16x3"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic (seeded phantom, motion, coils)",
        "config": {"workload": f"precision: {N}-node ellipsoid, POD rank 10, 3-D radial 256 x {args.spokes} "
                               f"samples (|k| <= 500 1/m), 8 coils, one frame per step",
                   "node_samples_per_step": units, "columns": C},
        "f32": {"ms_per_step": res["f32"], "value": units / (res["f32"] / 1e3)},
        "rel_l2_vs_fp64": {"bf16x3": fp64.rel_l2(outs["bf16x3"][idx], ref), "f32": fp64.rel_l2(outs["f32"][idx], ref),
                           "samples": int(args.check_samples)},
    }


# -------------------------------------------------------- serving (cfg 4) --

def build_serving_requests(n_requests: int, rate: float, seed: int = 5, max_nodes: int = 200_000,
                           max_samples: int = 262_144, max_frames: int = 4):
    """A Poisson request stream: meshes log-uniform in [10k, max_nodes] nodes,
    T1/T2 as in the plain configuration, Cartesian / radial / stack-of-spirals
    trajectories of 16k-max_samples samples, 1-8 coils, 1-max_frames frames
    with sinusoidal POD motion (rank 3) on every other request."""
    from feelmri_b200 import workloads as W
    from feelmri_b200.serving import Request
    rng = np.random.default_rng(seed)
    shapes = (W.cylinder, W.ellipsoid, W.tube)
    t = 0.0
    reqs = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n = int(np.exp(rng.uniform(np.log(1e4), np.log(max_nodes))))
        mesh = shapes[i % 3](n)
        N = mesh.n_nodes
        S = np.exp(rng.uniform(np.log(16384), np.log(max_samples)))
        kind = i % 3
        if kind == 0:
            n_kz = 16
            side = max(8, int(round(np.sqrt(S / n_kz))))
            traj = W.cartesian(res=(side, side, n_kz))
        elif kind == 1:
            n_sp = 512
            traj = W.radial3d(n_ro=max(8, int(round(S / n_sp))), n_spokes=n_sp, kmax=500.0)
        else:
            il, n_kz = 16, 16
            traj = W.spiral_stack(n_ro=max(16, int(round(S / (il * n_kz)))), n_interleaves=il, n_kz=n_kz)
        T1, T2 = W.tissue(N, seed + i)
        coils = W.coil_maps(mesh.nodes, int(rng.integers(1, 9)), seed=seed + i)
        pod = W.sinusoidal_pod(N, n_modes=3, amp=1e-3, period=800.0, n_frames=8, seed=seed + i) if i % 2 else None
        blocks = [W.hard_pulse_block(0.0, 15.0, 5.0, grad=((2.0, 0.0, 0.0), 1.0, 1.0)),
                  W.hard_pulse_block(5.0, 15.0, 5.0)]
        reqs.append(Request(rid=i, mesh=mesh, T1=T1, T2=T2, phi=W.off_resonance(N, 20.0, seed + i), blocks=blocks,
                            traj=traj, coils=coils, frames=int(rng.integers(1, max_frames + 1)), pod=pod,
                            arrival=t))
    return reqs


def run_serving(args) -> dict:
    """Requests arrive as a Poisson stream and are served continuously: each
    admitted request keeps its mesh, tissue, mass weights and magnetisation on
    the device and runs its frames on its own stream; requests are admitted as
    slots and HBM free up.  Reports latency percentiles and throughput."""
    import torch
    from feelmri_b200.serving import Server
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    reqs = build_serving_requests(args.requests, args.rate)
    build_s = time.perf_counter() - t0
    # warm-up: one small request through a server (kernels loaded, contexts made)
    Server(device=dev, slots=1).serve(build_serving_requests(1, args.rate, seed=99, max_nodes=12_000,
                                                             max_samples=20_000, max_frames=1), realtime=False)
    srv = Server(device=dev, slots=args.slots)
    t0 = time.perf_counter()
    items = srv.serve(reqs, realtime=True)
    wall = time.perf_counter() - t0
    stats = Server.summary(items)
    work = sum(it.req.work for it in items if it.error is None)
    return {
        "metric": METRIC, "value": work / wall, "unit": "node*k-sample/s", "n_gpus": 1, "steps": 1,
        "warmup": 1, "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic (seeded request stream)",
        "config": {"workload": f"serving: {len(reqs)} requests, Poisson arrivals at {args.rate} req/s, meshes "
                               "10k-200k nodes, Cartesian / radial / stack-of-spirals 16k-262k samples, 1-8 coils, "
                               "1-4 frames, POD motion on every other request",
                   "slots": args.slots, "node_samples": work},
        "latency_s": {k: stats[k] for k in ("p50_s", "p99_s", "mean_s", "max_s")},
        "requests": stats["requests"], "failed": stats["failed"],
        "setup_s": {"requests": build_s},
    }


def _lib_launches() -> int:
    from feelmri_b200 import _lib
    return _lib.launch_count()


def build_sequence_blocks(n_dummy: int, n_frames: int, spacing: float = 40.0, enc=(1, 0, 0)):
    """One encoding of the phase-contrast example's sequence
    (examples/phase_contrast.py:119-160): n_dummy unstored imaging blocks to
    reach the steady state, each followed by an empty spacing block (1 ms
    steps) up to `spacing` ms, then n_frames stored imaging blocks with their
    spacing blocks."""
    from feelmri_b200 import workloads as W
    blocks, t = [], 0.0
    for i in range(n_dummy + n_frames):
        b = W.pc_imaging_block(t, enc, venc=VENC)
        b.store_magnetization = i >= n_dummy
        dur = float(b.times[-1] - b.times[0])
        g = W.hard_pulse_block(t + dur, 0.0, spacing - dur, dt=1.0)
        g.empty = True
        blocks += [b, g]
        t += spacing
    return blocks


def run_sequence(args) -> dict:
    """BlochSolver over a whole encoding sequence through the public API:
    every block in one launch (the default) against the block-by-block loop
    (one solve per block, the reference's structure)."""
    import torch
    from feelmri_b200 import _lib, ops
    from feelmri_b200.Bloch import BlochSolver
    from feelmri_b200 import workloads as W
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    case = build_case(n_nodes=args.nodes)
    N = case["N"]
    nodes32 = case["mesh"].nodes.astype(np.float32)
    blocks = build_sequence_blocks(args.dummies, args.frames)
    node_steps = float(N) * sum(b.times.shape[0] - 1 for b in blocks)

    def solver(path):
        s = BlochSolver(blocks, nodes32, M0=1.0, T1=case["T1"], T2=case["T2"], delta_B=case["dB"], gamma=W.GAMMA,
                        pod_trajectory=case["vel"])
        if path == "blocks":
            s._solve_sequence = s._solve_blocks
        return s

    ctx = ops.ctx_for(dev)
    out = {}
    results = {}
    for path in ("sequence", "blocks"):
        for _ in range(max(3, args.warmup)):
            solver(path).solve()
        torch.cuda.synchronize()
        _lib.timing_reset(ctx)
        _lib.timing(ctx, True)
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            s = solver(path)
            m, z = s.solve()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        _lib.timing(ctx, False)
        k_ms, k_n = _lib.timing_query(ctx, "bloch")
        sec = statistics.median(ts)
        out[path] = {"value": node_steps / sec, "ms": sec * 1e3, "kernel_ms": k_ms / max(args.steps, 1),
                     "kernel_launches_per_solve": k_n / max(args.steps, 1)}
        results[path] = (m, z)
    same = all(np.array_equal(a, b) for a, b in zip(results["sequence"], results["blocks"]))
    return {"metric": "node-step/s (Bloch block sequence, public BlochSolver API)", "value": out["sequence"]["value"],
            "unit": "node-step/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out["sequence"]["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded tube, tissue and flow)",
            "config": {"workload": f"one phase-contrast encoding: {args.dummies} steady-state + {args.frames} stored "
                                   f"imaging blocks, each with a 1-ms-step spacing block (TR 40 ms), "
                                   f"{N // 1000}k-node tube with rank-1 flow POD",
                       "nodes": N, "blocks": len(blocks), "node_steps": node_steps,
                       "timer": "host wall clock around solver construction + solve(), device synchronised"},
            "block_loop": out["blocks"], "sequence": out["sequence"],
            "speedup_vs_block_loop": out["sequence"]["value"] / out["blocks"]["value"],
            "bit_identical_to_block_loop": bool(same)}


def run_pod_build(args) -> dict:
    """POD construction (Motion.POD) from displacement snapshots at the
    precision workload's scale: 500k nodes x 3 components x 40 frames,
    rank-10 fit.  numpy (the reference's computation) against
    backend="cuda" (snapshot products on the GPU), both end to end from host
    arrays, host clock."""
    import torch
    from feelmri_b200.Motion import POD
    rng = np.random.default_rng(6)
    P, t, r = args.nodes if args.nodes != N_NODES else 500_000, 40, 10
    times = np.linspace(0.0, 800.0, t)
    modes = rng.normal(0.0, 1e-3, (P, 3, r)).astype(np.float32)
    # distinct frequencies and decaying amplitudes: a well-separated rank-10 history
    freq, amp = np.arange(1, r + 1), 0.8 ** np.arange(r)
    w = (amp * np.sin(2 * np.pi * freq[None, :] * times[:, None] / 800.0 + rng.uniform(0, 6, r)[None, :])).astype(
        np.float32)
    data = np.einsum("pcm,tm->pct", modes, w).astype(np.float32)
    torch.cuda.init()
    POD(times[:4], data[:1000, :, :4], n_modes=2, backend="cuda")  # load the library, warm the context
    out = {}
    for backend in ("cuda", "numpy"):
        ts = []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            pod = POD(times, data, n_modes=r, backend=backend)
            ts.append(time.perf_counter() - t0)
        out[backend] = {"s": statistics.median(ts), "modes": pod.modes, "weights": pod.weights}
    errs = []
    for m in range(r):
        a, b = out["numpy"]["modes"][..., m], out["cuda"]["modes"][..., m]
        sgn = np.sign(np.vdot(a.ravel(), b.ravel()))
        errs.append(float(np.linalg.norm(a - sgn * b) / np.linalg.norm(a)))
    return {"metric": "POD construction time (Motion.POD, rank 10)", "value": out["cuda"]["s"], "unit": "s",
            "n_gpus": 1, "steps": args.steps, "warmup": 1, "ms_per_step": out["cuda"]["s"] * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32 data, f64 sums",
            "data": "synthetic rank-10 displacement snapshots",
            "config": {"workload": f"POD of {P} nodes x 3 x {t} frames, {r} modes", "timer": "host wall clock"},
            "numpy_s": out["numpy"]["s"], "speedup_vs_numpy": out["numpy"]["s"] / out["cuda"]["s"],
            "max_mode_rel_diff_vs_numpy": max(errs)}


def run_recon(args) -> dict:
    """Exact adjoint NUDFT (Recon.nudft_adjoint): 3-D radial k-space (256
    readout points x 1024 spokes, |k| <= 480 1/m) with 4 coils onto a
    96 x 96 x 32 voxel grid (FOV 0.2 x 0.2 x 0.0667 m, which covers the
    trajectory's extent in-plane), density-weighted by the radial ramp.  The
    adjoint runs as a Signal with the roles swapped, so the Cartesian voxel
    grid factors and the split-BF16 tensor-core form applies to any
    trajectory.  Split-BF16 against FP32, both checked against the FP64
    direct sum on 64 voxels."""
    import torch
    from feelmri_b200 import Recon, workloads as W
    from oracle import fp64
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    tr = W.radial3d(n_ro=256, n_spokes=1024, kmax=480.0)
    kx, ky, kz = tr.kx, tr.ky, tr.kz
    S, C = kx.size, 4
    rng = np.random.default_rng(8)
    K = ((rng.normal(size=(S, C)) + 1j * rng.normal(size=(S, C))) * 1e-3).astype(np.complex64)
    dcw = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2).reshape(-1).astype(np.float32) ** 2
    shape, fov = (96, 96, 32), (0.2, 0.2, 0.0667)
    res, imgs = {}, {}
    for prec in ("bf16x3", "f32"):
        for _ in range(max(1, args.warmup)):
            Recon.nudft_adjoint(K, kx, ky, kz, shape, fov, dcw=dcw, precision=prec)
        torch.cuda.synchronize()
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            imgs[prec] = Recon.nudft_adjoint(K, kx, ky, kz, shape, fov, dcw=dcw, precision=prec)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        res[prec] = statistics.median(ts)
    X, Y, Z = Recon.grid_points(shape, fov)
    pts = np.stack([X, Y, Z], -1).reshape(-1, 3)
    idx = np.random.default_rng(9).choice(pts.shape[0], 64, replace=False)
    ref = fp64.nudft_adjoint(kx, ky, kz, K, pts[idx], dcw=dcw)
    units = float(np.prod(shape)) * S
    return {"metric": "voxel*k-sample/s (exact adjoint NUDFT, public Recon API)", "value": units / res["bf16x3"],
            "unit": "voxel*k-sample/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res["bf16x3"] * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3", "data": "synthetic radial k-space",
            "config": {"workload": f"adjoint NUDFT: radial 256 x 1024 ({S} samples), {C} coils -> 96x96x32 grid",
                       "columns": C, "timer": "host wall clock around the call (host arrays in and out)"},
            "f32": {"ms_per_step": res["f32"] * 1e3, "value": units / res["f32"]},
            "rel_l2_vs_fp64": {"bf16x3": fp64.rel_l2(imgs["bf16x3"].reshape(-1, C)[idx], ref),
                               "f32": fp64.rel_l2(imgs["f32"].reshape(-1, C)[idx], ref), "voxels": 64}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="bf16x3", choices=["f32", "bf16x3"])
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--workload", default="phase_contrast",
                    choices=["phase_contrast", "batching", "serving", "precision", "sequence", "pod", "recon"],
                    help="phase_contrast: the metric's configuration; batching: many phantoms in one launch; "
                         "serving: a Poisson request stream; precision: radial, 8 coils, rank-10 motion")
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--spokes", type=int, default=4096)
    ap.add_argument("--check-samples", type=int, default=256)
    ap.add_argument("--phantoms", type=int, default=BATCH_PHANTOMS)
    ap.add_argument("--dummies", type=int, default=80, help="sequence workload: steady-state blocks")
    ap.add_argument("--frames", type=int, default=20, help="sequence workload: stored imaging blocks")
    ap.add_argument("--nodes", type=int, default=N_NODES,
                    help="mesh size (smaller cases of the same workload for profiling; the metric uses the default)")
    args = ap.parse_args()
    if args.impl == "reference":
        res = run_reference(args)
    elif args.workload == "batching":
        res = run_batching(args)
    elif args.workload == "serving":
        res = run_serving(args)
    elif args.workload == "precision":
        res = run_precision(args)
    elif args.workload == "sequence":
        res = run_sequence(args)
    elif args.workload == "pod":
        res = run_pod_build(args)
    elif args.workload == "recon":
        res = run_recon(args)
    else:
        res = run_gpu(args)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
