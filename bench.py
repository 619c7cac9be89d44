"""Benchmark of the simulation hot path on one node.

Default workload (the batched configuration, on which the split-BF16 >= 5x
FP32 target is stated): 64 phantoms of uneven size -- node counts
log-uniform in [5k, 300k], shapes cycling cylinder / ellipsoid / tube --
each with SPAMM tagging (two 90-degree pulses, 8 mm tags) then a 15-degree
GRE excitation, a per-phantom 3-D Cartesian grid or stack of spirals of
4k-200k samples and 1-2 Gaussian receive coils.

One step simulates one frame of every phantom: the fused Bloch sweeps of
both blocks (final states), the coil columns, then the mass-weighted NUDFT
of all 64 phantoms.  Units: node*k-sample = sum over phantoms of nodes x
k-space samples.  Two forms run in the same process:

* split-BF16 tensor-core form: ONE persistent launch for all 64 Signals
  (fm_signal_batch_enqueue) with work units picked by the autotuner;
* FP32 CUDA-core form (the drop-in form): one Signal launch per phantom.

`value` is the split-BF16 step, timed as a replay of the frame captured once
in a CUDA graph (every kernel of the frame runs in each replay; the
stream-launched steps, which give the kernel timings and the FP32 ratio, are
under `stream`); the FP32 step, their ratio, the FP64 check
of both forms, `e2e` (host arrays in, host arrays out, through
feelmri_b200.serving.simulate_batch), the Signal kernel's roofline and a
bounded CPU sample are in the same JSON line, and so are the other
configurations (plain FP64 20k-node GRE, phase-contrast flow, radial
precision frame, serving under a Poisson stream), each with its own clock
record.  Inputs are seeded synthetic stand-ins (the reference's phantoms are
not available).  With --gpus N each rank simulates its own batch of 64
phantoms (independent objects, weak scaling, no collective on the data
path).

  python bench.py [--gpus N] [--steps K] [--warmup W]
  python bench.py --impl reference ...   (the CPU restatement of the reference, bounded sample)
  python bench.py --workload {batching,plain,phase_contrast,precision,serving,sequence,pod,recon,node_partition}
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
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
BATCH_PHANTOMS = 64
FLUSH_BYTES = 512 << 20  # > 126 MB of L2


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




def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        d["source"] = "measured"
        return d
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


def cpu_info() -> dict:
    """CPU model, physical cores and the threads this process may use."""
    model, cores = None, set()
    try:
        for block in Path("/proc/cpuinfo").read_text().split("\n\n"):
            f = {}
            for line in block.splitlines():
                if ":" in line:
                    k, v = line.split(":", 1)
                    f[k.strip()] = v.strip()
            model = model or f.get("model name")
            if "core id" in f:
                cores.add((f.get("physical id", "0"), f["core id"]))
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count() or 1
    return {"model": model, "physical_cores": len(cores) or None, "logical_cpus": os.cpu_count(),
            "threads_usable": usable}


def _traffic_from_profile(name: str) -> float | None:
    """DRAM bytes per launch recorded in a committed ncu summary
    (profiles/<name>.md holds a line 'traffic_bytes_per_launch: <bytes>')."""
    p = ROOT / "profiles" / f"{name}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def _dist():
    """(rank, world, local rank, device, torch.distributed or None)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180), device_id=dev)
    return rank, world, local, dev, dist


def _max_over_ranks(dist, dev, value: float) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed_steps(fn, steps: int, warmup: int, dev, local: int, ctx, kernels=("signal_tc", "signal_f32"),
                dist=None, flush=None, nvtx: str = "step") -> dict:
    """W untimed steps, then K steps each bracketed by CUDA events on the
    launching stream, L2 flushed between them (outside the events), clocks
    sampled meanwhile, library kernel events on; barrier + synchronize on
    both sides; the total is the max over ranks."""
    import torch
    from feelmri_b200 import _lib
    stream = torch.cuda.current_stream(dev)
    ctxs = list(ctx) if isinstance(ctx, (list, tuple)) else [ctx]
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    for c in ctxs:
        _lib.timing_reset(c)
        _lib.timing(c, True)
    l0 = _lib.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize(dev)
        # an NVTX range marks the timed steps for a profiler (no cost without one)
        torch.cuda.nvtx.range_push(f"timed:{nvtx}")
        for a, b in ev:
            if flush is not None:
                flush.zero_()
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize(dev)
    launches = _lib.launch_count() - l0
    for c in ctxs:
        _lib.timing(c, False)
    if dist:
        dist.barrier()
    ms = [a.elapsed_time(b) for a, b in ev]
    total = _max_over_ranks(dist, dev, float(sum(ms)))
    out = {"ms_per_step": total / steps, "median_ms": statistics.median(ms), "total_ms": total,
           "steps": steps, "warmup": warmup, "launches": launches, "clocks": clk.summary()}
    def query(name):
        # summed over the contexts (the launch stream's and its helper streams')
        ms_n = [_lib.timing_query(c, name) for c in ctxs]
        return sum(m for m, _ in ms_n), sum(n for _, n in ms_n)
    for k in kernels:
        k_ms, k_n = query(k)
        if k_n:
            out[f"{k}_ms_per_launch"] = k_ms / k_n
            out[f"{k}_launches"] = k_n
    b_ms, b_n = query("bloch")
    # device time of the Bloch sweeps, summed over streams (they may overlap)
    out["bloch_ms_per_step"] = b_ms / steps
    return out


# ------------------------------------------------------ batching (cfg 3) --

def build_batch_requests(n_phantoms: int = BATCH_PHANTOMS, seed: int = 4):
    """Phantoms of uneven size: node counts log-uniform in [5k, 300k], shapes
    cycling cylinder / ellipsoid / tube; SPAMM tagging (8 mm) then a
    15-degree GRE excitation; per phantom a 3-D Cartesian grid or a stack of
    spirals of 4k-200k samples (log-uniform) and 1 or 2 receive coils.
    Returned as serving.Request objects (lumped mass weights included)."""
    from feelmri_b200 import workloads as W
    from feelmri_b200.Assemble import mass_lumped
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    from feelmri_b200.serving import Request
    rng = np.random.default_rng(seed)
    shapes = (W.cylinder, W.ellipsoid, W.tube)
    fe, qr = FiniteElement(), QuadratureRule(order=2)
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
        w = mass_lumped(mesh.elems, mesh.nodes, fe, qr).astype(np.float32)
        out.append(Request(rid=i, mesh=mesh, T1=T1, T2=T2, phi=W.off_resonance(N, 20.0, seed + i), blocks=blocks,
                           traj=traj, coils=coils, weights=w))
    return out


def _fp64_check(req, cols: np.ndarray, outs: dict, n_samples: int, seed: int) -> dict:
    """rel-L2 of each form's k-space against the FP64 oracle on a seeded
    subset of samples (float-rounded pi, the reference's convention)."""
    import scipy.sparse as sp
    from oracle import fp64
    t = req.traj
    S = t.n_samples
    idx = np.random.default_rng(seed).choice(S, min(S, n_samples), replace=False)
    ref = fp64.signal(sp.diags(req.weights.astype(np.float64)).tocsc(), t.kx, t.ky, t.kz, t.t,
                      req.mesh.nodes.astype(np.float32), req.phi, req.T2, cols, pi_mode="float", sample_idx=idx)
    return {k: fp64.rel_l2(v.reshape(S, -1)[idx], ref) for k, v in outs.items()}


def run_batching(args) -> dict | None:
    import torch
    from feelmri_b200 import _lib, autotune, ops
    from feelmri_b200.serving import Simulation, enqueue_bloch_all, helper_streams
    rank, world, local, dev, dist = _dist()
    t0 = time.perf_counter()
    reqs = build_batch_requests(args.phantoms, seed=4 + 1000 * rank)
    build_s = time.perf_counter() - t0
    sims = [Simulation(r, dev) for r in reqs]
    torch.cuda.synchronize(dev)
    units = float(sum(r.n_nodes * r.traj.n_samples for r in reqs))
    vwork = float(sum(r.n_nodes * r.traj.n_samples * r.n_coils for r in reqs))
    motions = [s.motion(0) for s in sims]
    problems = [(s.sig, m, s.out) for s, m in zip(sims, motions)]
    out32 = [torch.empty_like(s.out) for s in sims]

    zero_frames = [0] * len(sims)

    def bloch_all():
        enqueue_bloch_all(sims, zero_frames)

    bloch_all()
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    if args.tuning:
        sn, kc = (int(x) for x in args.tuning.split("/"))
        tuning, tried = ops.Tuning(split_nodes=sn, kz_cap=kc), {}
    else:
        tuning, tried = autotune.tune(problems, force=True)
    tune_s = time.perf_counter() - t1
    batch = ops.SignalBatch(problems, tuning)

    def step_tc():
        bloch_all()
        batch.enqueue()

    def step_32():
        bloch_all()
        for s, m, o in zip(sims, motions, out32):
            ops.signal(s.sig, m, "f32", out=o, sync=False)

    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    ctx = [ops.ctx_for(dev)]
    for st in helper_streams(dev):
        with torch.cuda.stream(st):
            ctx.append(ops.ctx_for(dev))
    tc = timed_steps(step_tc, args.steps, args.warmup, dev, local, ctx, dist=dist, flush=flush, nvtx="bf16x3")
    batch.status()
    f32_steps = max(3, min(args.steps, args.f32_steps))
    f32 = timed_steps(step_32, f32_steps, 2, dev, local, ctx, dist=dist, flush=flush, nvtx="f32")

    # The same split-BF16 step captured once in a CUDA graph.  The line's
    # timed steps replay it: every kernel of the frame (Bloch sweeps, run
    # building, classification, coil columns, the persistent Signal launch,
    # split sums) runs in each replay, without the per-launch host cost.
    # The stream-launched steps above give the kernel timings.
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        step_tc()
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        l0 = _lib.launch_count()
        with torch.cuda.graph(g, stream=stream):
            step_tc()
        graph_launches = _lib.launch_count() - l0
        tcg = timed_steps(g.replay, args.steps, args.warmup, dev, local, ctx, dist=dist, flush=flush,
                          nvtx="bf16x3_graph")
    stream.synchronize()
    del g

    # both forms on the same coil columns, checked against FP64
    bloch_all()
    batch.enqueue()
    for s, m, o in zip(sims, motions, out32):
        ops.signal(s.sig, m, "f32", out=o, sync=False)
    batch.status()
    torch.cuda.synchronize(dev)
    sizes = [r.n_nodes for r in reqs]
    pick = sorted({int(np.argmax(sizes)), int(np.argmin(sizes)), 1, 2})
    checks = {}
    for i in pick:
        checks[i] = _fp64_check(reqs[i], sims[i].cols.cpu().numpy(),
                                {"bf16x3": sims[i].out.cpu().numpy(), "f32": out32[i].cpu().numpy()},
                                args.check_samples, seed=i)

    result = None
    if rank == 0:
        peaks = _peaks()
        value = units * world / (tcg["ms_per_step"] / 1e3)
        k_ms = tc.get("signal_tc_ms_per_launch")
        flops = 3 * 8.0 * vwork  # split-BF16 MMA flops of the contraction: 3 products x 8 real flops per column
        achieved = flops / (k_ms / 1e3) / 1e12 if k_ms else None
        roof = {"bound": "tensor", "achieved": achieved, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                "frac": achieved / peaks["bf16_tflops"] if achieved else None,
                "frac_of_sustained": achieved / peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"])
                if achieved else None,
                "traffic": _traffic_from_profile("signal_tc_kernel__batching_64"), "traffic_unit": "bytes per launch",
                "kernel": "fm::signal_tc_kernel (one launch per step)", "kernel_ms": k_ms,
                "algorithmic_flops_per_launch": flops, "peak_source": f"{peaks['source']} (burst)"}
        result = {
            "metric": METRIC, "value": value, "unit": "node*k-sample/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tcg["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic (seeded phantoms, sequences and trajectories)",
            "config": {"workload": f"batching: {len(reqs)} phantoms per GPU, nodes log-uniform 5k-300k "
                                   f"(total {sum(sizes)}), SPAMM (8 mm) + 15-degree GRE, Cartesian or "
                                   "stack-of-spirals 4k-200k samples, 1-2 coils; one frame of every phantom "
                                   "per step (Bloch + coil columns + NUDFT)",
                       "node_samples_per_step_per_gpu": units, "phantoms": len(reqs),
                       "precision": "bf16x3 (split-BF16, one persistent launch for all phantoms)",
                       "l2": "flushed (512 MB write) between timed steps",
                       "step_form": "one CUDA-graph replay of the whole frame (every kernel runs each step)",
                       "parallelism": f"independent batches x{world}" if world > 1 else "single GPU"},
            "f32": {"value": units * world / (f32["ms_per_step"] / 1e3), "ms_per_step": f32["ms_per_step"],
                    "steps": f32["steps"], "warmup": f32["warmup"], "clocks": f32["clocks"],
                    "kernel_ms_per_launch": f32.get("signal_f32_ms_per_launch"),
                    "form": "FP32 CUDA-core Signal, one launch per phantom"},
            "speedup_vs_f32": f32["ms_per_step"] / tc["ms_per_step"],
            "speedup_vs_f32_form": "stream-launched steps of both forms",
            "stream": {"ms_per_step": tc["ms_per_step"], "steps": tc["steps"], "warmup": tc["warmup"],
                       "launches": int(tc["launches"]), "clocks": tc["clocks"]},
            "rel_l2_vs_fp64": {"bf16x3_max": max(c["bf16x3"] for c in checks.values()),
                               "f32_max": max(c["f32"] for c in checks.values()),
                               "phantoms_checked": pick, "samples_each": args.check_samples},
            "roofline": roof,
            "bloch_ms_per_step": tc["bloch_ms_per_step"],
            "graph_ms_per_step": tcg["ms_per_step"],
            "gpu_launches": int(graph_launches) * args.steps,
            "graph_launches_per_step": int(graph_launches),
            "clocks": tcg["clocks"],
            "tuning": {"split_nodes": tuning.split_nodes, "kz_cap": tuning.kz_cap, "search_s": tune_s,
                       "tried_ms": {f"{k.split_nodes}/{k.kz_cap}": v for k, v in tried.items()}},
            "setup_s": {"phantoms": build_s},
        }
        if args.e2e:
            result["e2e"] = run_batch_e2e(args, reqs, tuning, dev)
        if args.cpu_baseline and world == 1:
            result["cpu_baseline"] = cpu_sample(reqs, budget_s=args.cpu_seconds)
    del sims, problems, batch
    torch.cuda.empty_cache()
    if result is not None and world == 1 and args.extras:
        for name, fn in (("plain", run_plain), ("phase_contrast", run_phase_contrast),
                         ("precision", run_precision), ("serving", run_serving)):
            try:
                result[name] = fn(args, extra=True)
            except Exception as exc:  # noqa: BLE001 - an extra never hides the headline line
                result[name] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.empty_cache()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def run_batch_e2e(args, reqs, tuning, dev) -> dict:
    """The batched step through the public host-level call
    (serving.simulate_batch): every phantom's inputs go up from host memory
    through pinned staging, Bloch + coil columns + one persistent Signal
    launch run, and every k-space comes back to host memory.  Host wall
    clock around the call (it ends with the results on the host)."""
    import torch
    from feelmri_b200.serving import simulate_batch
    for _ in range(2):
        simulate_batch(reqs, dev, tuning)
    torch.cuda.synchronize(dev)
    n = max(3, min(args.steps, 5))
    ts = []
    for _ in range(n):
        t0 = time.perf_counter()
        ks = simulate_batch(reqs, dev, tuning)
        ts.append(time.perf_counter() - t0)
    units = float(sum(r.n_nodes * r.traj.n_samples for r in reqs))
    h2d = 0
    for r in reqs:
        t = r.traj
        h2d += r.mesh.n_nodes * 3 * 4 + 4 * r.n_nodes * 4 + r.coils.size * 8 + 4 * t.kx.size * 4
        h2d += sum(b.rf.size * 8 + b.G.size * 4 + b.dt.size * 4 for b in r.blocks)
    d2h = sum(k.nbytes for k in ks)
    sec = statistics.median(ts)
    return {"value": units / sec, "unit": "node*k-sample/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": sec * 1e3, "steps": n,
            "timer": "host wall clock around serving.simulate_batch (host arrays in, host arrays out)"}


# --------------------------------------------------- CPU sample (cfg 3) --

def _cpu_bloch_chunks(jobs, threads):
    """oracle.bloch_f32 (the reference's solve_mri loop, reference compiler
    flags) over independent node chunks on a thread pool (ctypes releases
    the GIL), like the reference's one-process-per-core node partition."""
    import oracle

    def run(job):
        nodes, T1, T2, blocks = job
        n = nodes.shape[0]
        m = np.zeros(n, np.complex64)
        z = np.ones(n, np.float32)
        dB = np.zeros(n, np.float32)
        from feelmri_b200.workloads import GAMMA
        for b in blocks:
            fm, fz = oracle.bloch_f32(nodes, T1, T2, dB, 1.0, np.float32(GAMMA), b.rf, b.G,
                                      b.dt.astype(np.float32), m, z, history=False, flavour="fast")
            m, z = (0 * fm).astype(np.complex64), fz
        return fm
    with ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(run, jobs))


def cpu_step(reqs, frac: float, threads: int) -> tuple[float, float, dict]:
    """One bounded CPU sample of the batched step: the Bloch sweeps of the
    first ceil(frac*N) nodes of every phantom, and every phantom's Signal
    (all nodes) over its first ceil(frac*n_ro) readout rows, so that Bloch
    and Signal keep the proportions of the full step.  Returns (node*k-samples,
    seconds, detail)."""
    import oracle
    import scipy.sparse as sp
    jobs = []
    for r in reqs:
        n = max(1, int(np.ceil(frac * r.n_nodes)))
        nodes = r.mesh.nodes[:n].astype(np.float32)
        per = max(1, n // threads)
        for a in range(0, n, per):
            jobs.append((nodes[a:a + per], r.T1[a:a + per], r.T2[a:a + per], r.blocks))
    t0 = time.perf_counter()
    _cpu_bloch_chunks(jobs, threads)
    t_bloch = time.perf_counter() - t0
    units = 0.0
    t0 = time.perf_counter()
    for r in reqs:
        t = r.traj
        rows = max(1, int(np.ceil(frac * t.shape[0])))
        sl = slice(0, rows)
        M = sp.diags(r.weights).tocsc()
        cols = (np.full((r.n_nodes, 1), 0.1 + 0.05j) * r.coils).astype(np.complex64)
        oracle.signal(M, t.kx[sl], t.ky[sl], t.kz[sl], t.t[sl], r.mesh.nodes.astype(np.float32), r.phi, r.T2, cols,
                      dtype=np.float32, threads=threads, flavour="fast")
        units += float(r.n_nodes) * t.kx[sl].size
    t_sig = time.perf_counter() - t0
    return units, t_bloch + t_sig, {"bloch_s": t_bloch, "signal_s": t_sig}


def _calibrate(reqs, threads, budget_s) -> float:
    frac = 0.002
    while True:
        _, sec, _ = cpu_step(reqs, frac, threads)
        if sec > 0.25 * budget_s or frac >= 1.0:
            break
        frac = min(1.0, frac * max(2.0, 0.5 * budget_s / max(sec, 1e-3)))
    return min(1.0, frac * budget_s / max(sec, 1e-3))


def cpu_sample(reqs, budget_s: float = 15.0) -> dict:
    """cpu_baseline of the default line: one bounded sample of the batched
    step on the host cores (the reference's loops restated in C, compiled with
    the reference's optimisation flags), sized to about budget_s seconds."""
    info = cpu_info()
    threads = info["threads_usable"]
    frac = _calibrate(reqs, threads, budget_s)
    units, sec, det = cpu_step(reqs, frac, threads)
    return {"value": units / sec, "unit": "node*k-sample/s", "cores": threads, "kind": "port",
            "sample": f"{frac:.4f} of the batched step: Bloch of the first {frac:.2%} of every phantom's nodes "
                      f"(both blocks) + every phantom's Signal over its first {frac:.2%} of readout rows "
                      f"(all nodes, all coils), {sec:.1f} s (Bloch {det['bloch_s']:.1f} s, Signal "
                      f"{det['signal_s']:.1f} s)",
            "cpu_model": info["model"], "physical_cores": info["physical_cores"],
            "implementation": "oracle/refsem.c (the reference's solve_mri / Signal loops restated), -O3 "
                              "-ffast-math, one thread per usable CPU over node ranges"}


def run_reference(args) -> dict | None:
    """The reference arm: the CPU restatement of the reference's path on the
    host cores, each step one bounded sample of the batched step (the same
    sample for every step); value, ms_per_step and steps describe exactly
    what ran."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    info = cpu_info()
    threads = info["threads_usable"]
    t0 = time.perf_counter()
    reqs = build_batch_requests_host(args.phantoms)
    build_s = time.perf_counter() - t0
    frac = _calibrate(reqs, threads, args.ref_step_seconds)
    for _ in range(args.warmup):
        cpu_step(reqs, frac, threads)
    secs, units = [], 0.0
    for _ in range(args.steps):
        units, sec, det = cpu_step(reqs, frac, threads)
        secs.append(sec)
    total = sum(secs)
    value = units * len(secs) / total
    full_units = float(sum(r.n_nodes * r.traj.n_samples for r in reqs))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    sample = (f"{frac:.4f} of the batched step per step: Bloch of the first {frac:.2%} of every phantom's nodes "
              f"+ every phantom's Signal over its first {frac:.2%} of readout rows (all nodes, all coils)")
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "node*k-sample/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / len(secs) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded phantoms, sequences and trajectories)",
            "config": {"workload": f"batching: {len(reqs)} phantoms, nodes log-uniform 5k-300k, SPAMM (8 mm) + "
                                   "15-degree GRE, Cartesian or stack-of-spirals 4k-200k samples, 1-2 coils",
                       "implementation": "CPU restatement of the reference's solve_mri and Signal loops "
                                         "(oracle/refsem.c, -O3 -ffast-math); the reference's own native modules "
                                         "cannot be built (baseline/_ref absent: Eigen is fetched from the network "
                                         "at configure time and pip install stops at metadata generation)",
                       "node_samples_per_step": units},
            "cpu_baseline": {"value": value, "unit": "node*k-sample/s", "cores": threads, "kind": "port",
                             "sample": sample, "cpu_model": info["model"],
                             "physical_cores": info["physical_cores"]},
            "full_step_equivalent_ms": full_units / value * 1e3,
            "setup_s": {"phantoms": build_s},
            "e2e": {"value": value, "unit": "node*k-sample/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def build_batch_requests_host(n_phantoms: int):
    """build_batch_requests without a GPU: the lumped weights by the oracle's
    exact P1 rule (volume / 4 per vertex)."""
    from feelmri_b200 import workloads as W
    from feelmri_b200.serving import Request
    from oracle import fp64
    rng = np.random.default_rng(4)
    shapes = (W.cylinder, W.ellipsoid, W.tube)
    out = []
    for i in range(n_phantoms):
        n = int(np.exp(rng.uniform(np.log(5e3), np.log(3e5))))
        mesh = shapes[i % 3](n)
        N = mesh.n_nodes
        T1, T2 = W.tissue(N, 4 + i)
        s_target = np.exp(rng.uniform(np.log(4e3), np.log(2e5)))
        n_kz = int(rng.choice([8, 16, 32]))
        if i % 2 == 0:
            side = max(4, int(round(np.sqrt(s_target / n_kz))))
            traj = W.cartesian(res=(side, side, n_kz))
        else:
            il = int(rng.choice([8, 16, 32]))
            n_ro = max(16, int(round(s_target / (il * n_kz))))
            traj = W.spiral_stack(n_ro=n_ro, n_interleaves=il, n_kz=n_kz)
        coils = W.coil_maps(mesh.nodes, int(rng.integers(1, 3)), seed=4 + i)
        blocks = [W.spamm_block(0.0), W.hard_pulse_block(3.0, 15.0, 5.0)]
        w = fp64.lumped_p1(mesh.elems, mesh.nodes).astype(np.float32)
        out.append(Request(rid=i, mesh=mesh, T1=T1, T2=T2, phi=W.off_resonance(N, 20.0, 4 + i), blocks=blocks,
                           traj=traj, coils=coils, weights=w))
    return out


# ------------------------------------------------------------ plain (cfg 0) --

def run_plain(args, extra: bool = False) -> dict:
    """The plain configuration at full size: a ~20k-node P1 cylinder (radius
    40 mm, height 80 mm, in a 0.1 m box), M0 = 1, T1 ~ U[0.8, 1.2] s,
    T2 ~ U[50, 100] ms, lumped mass weights, a spoiled GRE of 20 pulses of
    15 degrees at TR 5 ms, a 2-D Cartesian 64 x 64 readout and one coil;
    complex FP64 k-space through the FP64 Signal overload.  One step is the
    public API end to end from host arrays: BlochSolver (20 blocks, one
    sweep) then MRI.Signal with float64 arrays (the FP64 kernel).  The whole
    step also runs on the host cores through the CPU restatement, at full
    size."""
    import scipy.sparse as sp
    import torch
    import oracle
    from oracle import fp64
    from feelmri_b200 import _lib, ops
    from feelmri_b200 import workloads as W
    from feelmri_b200.Assemble import mass_lumped
    from feelmri_b200.Bloch import BlochSolver
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    from feelmri_b200.MRI import Signal
    dev = torch.device("cuda", torch.cuda.current_device())
    mesh = W.cylinder(20_000)
    N = mesh.n_nodes
    T1, T2 = W.tissue(N, 0)
    blocks = W.spoiled_gre(20, 15.0, 5.0)
    traj = W.cartesian(res=(64, 64, 1), fov=(0.1, 0.1, 0.1))
    S = traj.n_samples
    w = mass_lumped(mesh.elems, mesh.nodes, FiniteElement(), QuadratureRule(order=2))  # float64 nodes: float64
    M = sp.diags(np.asarray(w, np.float64)).tocsc()
    nodes64 = np.ascontiguousarray(mesh.nodes, np.float64)
    pts64 = [np.asarray(p, np.float64) for p in traj.points]
    t64 = np.asarray(traj.t, np.float64)
    phi64 = np.zeros(N)
    T2_64 = np.asarray(T2, np.float64)

    def step():
        s = BlochSolver(blocks, mesh.nodes.astype(np.float32), None, 1.0, T1, T2)
        m, _ = s.solve()
        return Signal(0, M, pts64, t64, nodes64, phi64, T2_64, m[:, -1:].astype(np.complex128), None)

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    ctx = ops.ctx_for(dev)
    steps = 5 if extra else args.steps
    _lib.timing_reset(ctx)
    _lib.timing(ctx, True)
    ts = []
    with ClockSampler(dev.index or 0) as clk:
        for _ in range(steps):
            t0 = time.perf_counter()
            K = step()
            ts.append(time.perf_counter() - t0)
    _lib.timing(ctx, False)
    sig_ms, sig_n = _lib.timing_query(ctx, "signal_f64")
    bl_ms, bl_n = _lib.timing_query(ctx, "bloch")
    sec = statistics.median(ts)
    m, _ = BlochSolver(blocks, mesh.nodes.astype(np.float32), None, 1.0, T1, T2).solve()
    Mxy = m[:, -1:]
    ref = fp64.signal(M, *pts64, t64, nodes64, phi64, T2_64, Mxy.astype(np.complex128), pi_mode="float")
    forms = {"f64": K}
    for prec in ("f32", "bf16x3"):
        forms[prec] = Signal(0, M.astype(np.float32), traj.points, traj.t, mesh.nodes.astype(np.float32),
                             phi64.astype(np.float32), T2, Mxy, None, precision=prec)
    rel = {k: fp64.rel_l2(v.reshape(S, -1), ref.reshape(S, -1)) for k, v in forms.items()}
    # the same step on the host cores, full size (CPU restatement)
    info = cpu_info()
    threads = info["threads_usable"]
    nodes32 = mesh.nodes.astype(np.float32)
    t0 = time.perf_counter()
    per = max(1, -(-N // threads))
    jobs = [(nodes32[a:a + per], T1[a:a + per], T2[a:a + per], blocks) for a in range(0, N, per)]
    with ThreadPoolExecutor(max_workers=threads) as ex:
        def run(job):
            n = job[0].shape[0]
            mm, zz = np.zeros(n, np.complex64), np.ones(n, np.float32)
            for b in blocks:
                fm, fz = oracle.bloch_f32(job[0], job[1], job[2], np.zeros(n, np.float32), 1.0, np.float32(W.GAMMA),
                                          b.rf, b.G, b.dt.astype(np.float32), mm, zz, history=False, flavour="fast")
                mm, zz = (0 * fm).astype(np.complex64), fz
            return fm
        last = np.concatenate(list(ex.map(run, jobs)))
    t_bloch = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.signal(M, *pts64, t64, nodes64, phi64, T2_64, last[:, None].astype(np.complex128), dtype=np.float64,
                  threads=threads, flavour="fast")
    t_sig = time.perf_counter() - t0
    units = float(N) * S
    return {"workload": f"plain: {N}-node P1 cylinder, spoiled GRE 20 x 15 deg TR 5 ms, 2-D Cartesian 64x64, "
                        "1 coil, complex FP64 k-space (FP64 Signal overload)",
            "metric": METRIC, "value": units / sec, "ms_per_step": sec * 1e3, "steps": steps, "warmup": 3,
            "timer": "host wall clock around BlochSolver + MRI.Signal (host arrays in and out)",
            "kernels_ms_per_step": {"bloch": bl_ms / steps, "signal_f64": sig_ms / max(sig_n, 1)},
            "rel_l2_vs_fp64_oracle": rel,
            "cpu_full_size": {"ms": (t_bloch + t_sig) * 1e3, "bloch_ms": t_bloch * 1e3, "signal_ms": t_sig * 1e3,
                              "value": units / (t_bloch + t_sig), "cores": threads, "kind": "port",
                              "sample": "the whole step at full size (no extrapolation)",
                              "cpu_model": info["model"]},
            "gpu_vs_cpu_full_size": (t_bloch + t_sig) / sec,
            "clocks": clk.summary()}


# --------------------------------------------------- phase contrast (cfg 1) --

def build_case(seed: int = 0, n_nodes: int = N_NODES):
    """Host-side synthetic inputs of the phase-contrast configuration."""
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


def run_phase_contrast(args, extra: bool = False) -> dict:
    """Phase-contrast flow: a 200k-node P1 tube (radius 12 mm, length 100 mm)
    with Poiseuille flow (peak 1 m/s) moving the nodes as a rank-1 velocity
    mode, off-resonance ~N(0, 20 Hz), a 3-D Cartesian 96 x 96 x 32 readout
    (96 distinct times) and 4 velocity encodings (VENC 1.5 m/s).  One step:
    4 fused Bloch sweeps of the imaging block, then the NUDFT of the 4
    encodings at once (V = 4), device-resident; split-BF16 and FP32 forms,
    each checked against FP64 on 256 seeded samples."""
    import scipy.sparse as sp
    import torch
    from oracle import fp64
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    from feelmri_b200.Assemble import mass_lumped
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    from feelmri_b200.MRI import signal_call_times
    from feelmri_b200 import workloads as W
    dev = torch.device("cuda", torch.cuda.current_device())
    case = build_case(n_nodes=args.nodes)
    N, traj, vel = case["N"], case["traj"], case["vel"]
    S, V = traj.n_samples, len(W.PC_ENCODINGS)
    w = mass_lumped(case["mesh"].elems, case["mesh"].nodes, FiniteElement(), QuadratureRule(order=2))
    up = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)  # noqa
    r0 = up(case["mesh"].nodes.astype(np.float32))
    T1, T2, dB = up(case["T1"]), up(case["T2"]), up(case["dB"])
    blocks = [(up(b.rf, torch.complex64), up(b.G), up(b.dt.astype(np.float32)), b.t0) for b in case["blocks"]]
    idx = torch.arange(N + 1, dtype=torch.int32, device=dev)
    Minds = ops.SparseCSC((N, N), idx, idx[:N], up(w.astype(np.float32)))
    sig = ops.SignalInputs(M=Minds, kx=up(traj.kx), ky=up(traj.ky), kz=up(traj.kz), t=up(traj.t), r0=r0,
                           phi=up(case["phi"]), T2=T2, Mxy=torch.empty((N, V), dtype=torch.complex64, device=dev))
    Mz_tmp = torch.empty((N,), dtype=torch.float32, device=dev)
    zero_m = torch.zeros((N,), dtype=torch.complex64, device=dev)
    one_z = torch.ones((N,), dtype=torch.float32, device=dev)
    outs = {p: torch.empty((*traj.shape, V), dtype=torch.complex64, device=dev) for p in ("bf16x3", "f32")}
    motions = []
    for rf, G, dt, t0 in blocks:
        vel.update_timeshift(t0)
        motions.append(lower(vel, N, dev))
    vel.update_timeshift(0.0)
    sig_motion = lower(vel, N, dev)

    def make_step(prec):
        def step():
            for e, (rf, G, dt, t0) in enumerate(blocks):
                inp = ops.BlochInputs(r0=r0, T1=T1, T2=T2, delta_B=dB, M0=1.0, gamma=W.GAMMA, rf=rf, G=G, dt=dt,
                                      Mxy0=zero_m, Mz0=one_z)
                ops.bloch_solve(inp, motions[e], history=False, Mxy_final=sig.Mxy[:, e], Mz_final=Mz_tmp)
            ops.signal(sig, sig_motion, prec, out=outs[prec], sync=False)
        return step

    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    ctx = ops.ctx_for(dev)
    steps = min(args.steps, 10) if extra else args.steps
    res = {p: timed_steps(make_step(p), steps, 3, dev, dev.index or 0, ctx, flush=flush) for p in ("bf16x3", "f32")}
    torch.cuda.synchronize(dev)
    # FP64 check of both forms on the same Mxy columns
    make_step("bf16x3")()
    ops.signal(sig, sig_motion, "f32", out=outs["f32"], sync=False)
    torch.cuda.synchronize(dev)
    Mxy_host = sig.Mxy.cpu().numpy()
    pick = np.random.default_rng(0).choice(S, args.check_samples, replace=False)
    run_times = signal_call_times(traj.t)[1:]
    disp = np.stack([vel(float(t)) for t in run_times])
    ref = fp64.signal(sp.diags(w).tocsc(), traj.kx, traj.ky, traj.kz, traj.t, case["mesh"].nodes.astype(np.float32),
                      case["phi"], case["T2"], Mxy_host, disp=disp, pi_mode="float", sample_idx=pick)
    rel = {p: fp64.rel_l2(outs[p].cpu().numpy().reshape(S, V)[pick], ref) for p in outs}
    peaks = _peaks()
    k_ms = res["bf16x3"].get("signal_tc_ms_per_launch")
    flops = 3 * 8.0 * V * float(N) * S
    units = float(N) * S
    return {"workload": f"phase-contrast flow: {N}-node P1 tube, Poiseuille 1 m/s, 96x96x32 Cartesian, "
                        "4 velocity encodings (VENC 1.5 m/s), off-resonance N(0,20 Hz); one frame per step",
            "metric": METRIC, "value": units / (res["bf16x3"]["ms_per_step"] / 1e3),
            "ms_per_step": res["bf16x3"]["ms_per_step"], "steps": steps, "warmup": 3,
            "f32": {"value": units / (res["f32"]["ms_per_step"] / 1e3), "ms_per_step": res["f32"]["ms_per_step"],
                    "kernel_ms": res["f32"].get("signal_f32_ms_per_launch"), "clocks": res["f32"]["clocks"]},
            "speedup_vs_f32": res["f32"]["ms_per_step"] / res["bf16x3"]["ms_per_step"],
            "rel_l2_vs_fp64": dict(rel, samples=int(args.check_samples)),
            "roofline": {"bound": "tensor", "kernel": "fm::signal_tc_kernel", "kernel_ms": k_ms,
                         "achieved": flops / (k_ms / 1e3) / 1e12 if k_ms else None, "unit": "TFLOP/s",
                         "peak": peaks["bf16_tflops"],
                         "frac": flops / (k_ms / 1e3) / 1e12 / peaks["bf16_tflops"] if k_ms else None,
                         "traffic": _traffic_from_profile("signal_tc_kernel__phase_contrast_200k")},
            "bloch_ms_per_step": res["bf16x3"]["bloch_ms_per_step"],
            "bloch_history_roofline": _bloch_history_roofline(r0, T1, T2, dB, blocks[1], vel, N, dev, flush, peaks),
            "clocks": res["bf16x3"]["clocks"]}


def _bloch_history_roofline(r0, T1, T2, dB, block, vel, N, dev, flush, peaks) -> dict:
    """The API-exact history form of one encoding block timed alone:
    algorithmic bytes = N n_t 12 written + N 48 read + n_t 24."""
    import torch
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    from feelmri_b200 import workloads as W
    rf, G, dt, t0 = block
    vel.update_timeshift(t0)
    motion = lower(vel, N, dev)
    zero_m = torch.zeros((N,), dtype=torch.complex64, device=dev)
    one_z = torch.ones((N,), dtype=torch.float32, device=dev)
    inp = ops.BlochInputs(r0=r0, T1=T1, T2=T2, delta_B=dB, M0=1.0, gamma=W.GAMMA, rf=rf, G=G, dt=dt,
                          Mxy0=zero_m, Mz0=one_z)
    ops.bloch_solve(inp, motion, history=True)
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(5):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ops.bloch_solve(inp, motion, history=True)
        b.record()
        b.synchronize()
        ms.append(a.elapsed_time(b))
    n_t = int(rf.shape[0])
    byt = float(N) * n_t * 12 + float(N) * 48 + n_t * 24
    med = statistics.median(ms)
    ach = byt / (med / 1e3) / 1e9
    return {"bound": "hbm", "ms": med, "bytes": byt, "achieved": ach, "unit": "GB/s", "peak": peaks["hbm_gbs"],
            "frac": ach / peaks["hbm_gbs"], "node_steps_per_s": float(N) * n_t / (med / 1e3), "n_t": n_t,
            "traffic": _traffic_from_profile("bloch_kernel__phase_contrast_200k")}


# ------------------------------------------------------ precision (cfg 2) --

def run_precision(args, extra: bool = False) -> dict:
    """Ellipsoid phantom (semi-axes 60/50/40 mm, ~500k nodes), POD motion
    (rank 10, Phi ~ N(0, 1 mm), sinusoidal weights, 800 ms cycle), 3-D radial
    readout (256 readout points x 4096 spokes, |k| <= 500 1/m, one distinct
    time per readout point), 8 Gaussian receive coils; one frame per step (the
    Signal of all coils after a 15-degree excitation).  Split-BF16 and FP32
    forms, each against the FP64 oracle on a seeded subset of samples."""
    import scipy.sparse as sp
    import torch
    from oracle import fp64
    from feelmri_b200 import ops
    from feelmri_b200._motion import lower
    from feelmri_b200.Assemble import mass_lumped
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    from feelmri_b200.MRI import signal_call_times
    from feelmri_b200 import workloads as W
    dev = torch.device("cuda", torch.cuda.current_device())
    mesh = W.ellipsoid(500_000 if args.nodes == N_NODES else args.nodes)
    N = mesh.n_nodes
    traj = W.radial3d(n_ro=256, n_spokes=args.spokes, kmax=500.0)
    S, C = traj.n_samples, 8
    T1, T2 = W.tissue(N, 2)
    phi = W.off_resonance(N, 20.0, 2)
    coils = W.coil_maps(mesh.nodes, C, seed=3)
    pod = W.sinusoidal_pod(N, n_modes=10, amp=1e-3, period=800.0, n_frames=20, seed=2)
    w = mass_lumped(mesh.elems, mesh.nodes, FiniteElement(), QuadratureRule(order=2))
    up = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)  # noqa
    idx = torch.arange(N + 1, dtype=torch.int32, device=dev)
    M = ops.SparseCSC((N, N), idx, idx[:N], up(w.astype(np.float32)))
    m0 = np.full(N, np.sin(np.deg2rad(15.0)), np.complex64)
    cols = up(m0[:, None] * coils, torch.complex64)
    sig = ops.SignalInputs(M=M, kx=up(traj.kx), ky=up(traj.ky), kz=up(traj.kz), t=up(traj.t), r0=up(
        mesh.nodes.astype(np.float32)), phi=up(phi), T2=up(T2), Mxy=cols)
    steps = 2 if extra else args.steps
    warm = 1 if extra else args.warmup
    res, outs, clocks = {}, {}, {}
    frame = [0]
    for prec in ("bf16x3", "f32"):
        out = torch.empty((*traj.shape, C), dtype=torch.complex64, device=dev)
        ms = []
        with ClockSampler(dev.index or 0) as clk:
            for f in range(warm + steps):
                pod.update_timeshift(40.0 * f)
                mo = lower(pod, N, dev)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                ops.signal(sig, mo, prec, out=out)
                b.record()
                b.synchronize()
                if f >= warm:
                    ms.append(a.elapsed_time(b))
                frame[0] = f
        res[prec] = statistics.median(ms)
        outs[prec] = out.cpu().numpy().reshape(S, C)
        clocks[prec] = clk.summary()
    pod.update_timeshift(40.0 * frame[0])
    pick = np.random.default_rng(2).choice(S, args.check_samples, replace=False)
    times = signal_call_times(traj.t)[1:]

    class _RunDisp:  # displacement of run g, computed only for the runs the subset touches
        def __getitem__(self, g):
            return pod(float(times[g]))

    ref = fp64.signal(sp.diags(w).tocsc(), traj.kx, traj.ky, traj.kz, traj.t, mesh.nodes.astype(np.float32), phi, T2,
                      cols.cpu().numpy(), disp=_RunDisp(), pi_mode="float", sample_idx=pick)
    units = float(N) * S
    rel = {p: fp64.rel_l2(outs[p][pick], ref) for p in outs}
    return {"workload": f"precision: {N}-node ellipsoid, POD rank 10, 3-D radial 256 x {args.spokes} samples "
                        f"(|k| <= 500 1/m), 8 coils, one frame per step",
            "metric": METRIC, "value": units / (res["bf16x3"] / 1e3), "ms_per_step": res["bf16x3"],
            "steps": steps, "warmup": warm, "columns": C,
            "f32": {"value": units / (res["f32"] / 1e3), "ms_per_step": res["f32"], "clocks": clocks["f32"]},
            "speedup_vs_f32": res["f32"] / res["bf16x3"],
            "rel_l2_vs_fp64": dict(rel, samples=int(args.check_samples),
                                   f32_over_bf16x3=rel["f32"] / rel["bf16x3"] if rel["bf16x3"] else None),
            "clocks": clocks["bf16x3"]}


# -------------------------------------------------------- serving (cfg 4) --

def build_serving_requests(n_requests: int, rate: float, seed: int = 5, max_nodes: int = 200_000,
                           max_samples: int = 262_144, max_frames: int = 4, min_nodes: int = 10_000,
                           min_samples: int = 16_384):
    """A Poisson request stream: meshes log-uniform in [min_nodes,
    max_nodes] nodes, T1/T2 as in the plain configuration, Cartesian / radial
    / stack-of-spirals trajectories of min_samples-max_samples samples, 1-8
    coils, 1-max_frames frames with sinusoidal POD motion (rank 3) on every
    other request."""
    from feelmri_b200 import workloads as W
    from feelmri_b200.serving import Request
    rng = np.random.default_rng(seed)
    shapes = (W.cylinder, W.ellipsoid, W.tube)
    t = 0.0
    reqs = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n = int(np.exp(rng.uniform(np.log(min_nodes), np.log(max_nodes))))
        mesh = shapes[i % 3](n)
        N = mesh.n_nodes
        S = np.exp(rng.uniform(np.log(min_samples), np.log(max_samples)))
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


def run_serving(args, extra: bool = False) -> dict:
    """A Poisson stream of simulation requests served with continuous
    batching: every in-flight request advances one frame per iteration, all
    of their Signals in one persistent launch; arrivals join the next launch.
    Reports latency percentiles and throughput, and the same requests served
    all at once against the sum of their solo service times (the overlap)."""
    import torch
    from feelmri_b200.serving import Server
    dev = torch.device("cuda", torch.cuda.current_device())
    t0 = time.perf_counter()
    n = args.requests
    reqs = build_serving_requests(n, args.rate)
    if args.full_sizes:
        # a few requests at the configuration's largest sizes (1M nodes, 2M samples, 30 frames)
        reqs += build_serving_requests(2, args.rate, seed=55, min_nodes=900_000, max_nodes=1_000_000,
                                       min_samples=1_900_000, max_samples=2_000_000, max_frames=30)
    build_s = time.perf_counter() - t0
    warm = build_serving_requests(2, args.rate, seed=99, max_nodes=12_000, max_samples=20_000, max_frames=1)
    Server(device=dev, slots=2).serve(warm, realtime=False)
    # each request alone (service time with nothing else on the GPU)
    alone = {}
    for r in reqs:
        (it,) = Server(device=dev, slots=1).serve([r], realtime=False)
        alone[r.rid] = it
    solo = [it.finished for it in alone.values()]
    # all at once: one mix, admitted together
    srv = Server(device=dev, slots=args.slots)
    t1 = time.perf_counter()
    mixed = srv.serve(reqs, realtime=False)
    mix_span = time.perf_counter() - t1
    same = all(it.error is None and np.array_equal(it.kspace, alone[it.req.rid].kspace) for it in mixed)
    # the Poisson stream in real time
    srv = Server(device=dev, slots=args.slots)
    with ClockSampler(dev.index or 0) as clk:
        t1 = time.perf_counter()
        items = srv.serve(reqs, realtime=True)
        wall = time.perf_counter() - t1
    stats = Server.summary(items)
    work = sum(it.req.work for it in items if it.error is None)
    return {"workload": f"serving: {len(reqs)} requests, Poisson arrivals at {args.rate} req/s, meshes 10k-"
                        f"{'1M' if args.full_sizes else '200k'} nodes, Cartesian / radial / stack-of-spirals "
                        f"16k-{'2M' if args.full_sizes else '262k'} samples, 1-8 coils, "
                        f"1-{30 if args.full_sizes else 4} frames, POD motion on every other request",
            "metric": METRIC, "value": work / wall, "ms_per_step": wall * 1e3, "slots": args.slots,
            "latency_s": {k: stats[k] for k in ("p50_s", "p99_s", "mean_s", "max_s")},
            "requests": stats["requests"], "failed": stats["failed"],
            "max_requests_per_launch": stats["max_requests_per_launch"],
            "overlap": {"all_at_once_span_s": mix_span, "sum_of_solo_s": float(sum(solo)),
                        "speedup": float(sum(solo)) / mix_span if mix_span > 0 else None,
                        "identical_alone_and_mixed": bool(same)},
            "setup_s": {"requests": build_s}, "clocks": clk.summary()}


# --------------------------------------------- node partition (multi-GPU) --

def run_node_partition(args) -> dict | None:
    """The reference's multi-rank scheme (Phantom.py:194-239,
    MPIUtilities.py:13-26) on GPUs: the phase-contrast tube's elements are
    split into one part per rank, each rank simulates its local nodes (lumped
    mass of its own elements, Bloch of its nodes, split-BF16 Signal of all
    samples) and the partial k-spaces are summed onto rank 0 by one NCCL
    reduce of the device buffer.  Total work is fixed: strong scaling."""
    import torch
    from feelmri_b200 import distributed as D, ops
    from feelmri_b200._motion import lower
    from feelmri_b200.Assemble import mass_lumped
    from feelmri_b200.FiniteElements import FiniteElement, QuadratureRule
    from feelmri_b200 import workloads as W
    from feelmri_b200.motion import SplineMotion
    rank, world, local, dev, dist = _dist()
    case = build_case(n_nodes=args.nodes)
    mesh, traj = case["mesh"], case["traj"]
    part = D.distribute_mesh(mesh.elems, mesh.nodes, world, rank)
    l2g = part.local_to_global
    N = l2g.size
    S, V = traj.n_samples, len(W.PC_ENCODINGS)
    w = mass_lumped(part.elems, part.nodes, FiniteElement(), QuadratureRule(order=2))
    term = case["vel"].terms[0]
    vel = SplineMotion.from_samples(term.modes[l2g], np.linspace(0.0, 1000.0, 20).astype(np.float32),
                                    np.ones((20, 1)), periodic=True, velocity=True)
    up = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)  # noqa
    r0 = up(part.nodes.astype(np.float32))
    T1, T2 = up(case["T1"][l2g]), up(case["T2"][l2g])
    dB = torch.zeros(N, dtype=torch.float32, device=dev)
    blocks = [(up(b.rf, torch.complex64), up(b.G), up(b.dt.astype(np.float32)), b.t0) for b in case["blocks"]]
    idx = torch.arange(N + 1, dtype=torch.int32, device=dev)
    sig = ops.SignalInputs(M=ops.SparseCSC((N, N), idx, idx[:N], up(w.astype(np.float32))), kx=up(traj.kx),
                           ky=up(traj.ky), kz=up(traj.kz), t=up(traj.t), r0=r0, phi=up(case["phi"][l2g]), T2=T2,
                           Mxy=torch.empty((N, V), dtype=torch.complex64, device=dev))
    zero_m = torch.zeros(N, dtype=torch.complex64, device=dev)
    one_z = torch.ones(N, dtype=torch.float32, device=dev)
    Mz_tmp = torch.empty(N, dtype=torch.float32, device=dev)
    out = torch.empty((*traj.shape, V), dtype=torch.complex64, device=dev)
    motions = []
    for rf, G, dt, t0 in blocks:
        vel.update_timeshift(t0)
        motions.append(lower(vel, N, dev))
    vel.update_timeshift(0.0)
    sig_motion = lower(vel, N, dev)

    def step():
        for e, (rf, G, dt, t0) in enumerate(blocks):
            inp = ops.BlochInputs(r0=r0, T1=T1, T2=T2, delta_B=dB, M0=1.0, gamma=W.GAMMA, rf=rf, G=G, dt=dt,
                                  Mxy0=zero_m, Mz0=one_z)
            ops.bloch_solve(inp, motions[e], history=False, Mxy_final=sig.Mxy[:, e], Mz_final=Mz_tmp)
        ops.signal(sig, sig_motion, "bf16x3", out=out, sync=False)
        return D.gather_data(out, group=None) if dist else out

    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    r = timed_steps(step, args.steps, args.warmup, dev, local, ops.ctx_for(dev), dist=dist, flush=flush)
    result = None
    if rank == 0:
        units = float(case["N"]) * S
        result = {"metric": METRIC, "value": units / (r["ms_per_step"] / 1e3), "unit": "node*k-sample/s",
                  "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                  "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "bf16x3",
                  "data": "synthetic (seeded mesh, tissue, flow and trajectory)",
                  "config": {"workload": f"node partition: phase-contrast tube ({case['N']} nodes) split over "
                                         f"{world} ranks by element, partial k-spaces summed onto rank 0 by NCCL "
                                         "reduce", "local_nodes_rank0": N, "parallelism": f"node partition x{world}"},
                  "gpu_launches": int(r["launches"]), "clocks": r["clocks"]}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result

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
    """POD construction from displacement snapshots at the precision
    workload's scale: 500k nodes x 3 components x 40 frames, rank-10 fit.
    The method of snapshots in numpy against snapshot_pod (the two products
    on the GPU), both from host arrays, host clock."""
    import torch
    from feelmri_b200.motion import snapshot_pod
    rng = np.random.default_rng(6)
    P, t, r = args.nodes if args.nodes != N_NODES else 500_000, 40, 10
    times = np.linspace(0.0, 800.0, t)
    modes = rng.normal(0.0, 1e-3, (P, 3, r)).astype(np.float32)
    freq, amp = np.arange(1, r + 1), 0.8 ** np.arange(r)
    w = (amp * np.sin(2 * np.pi * freq[None, :] * times[:, None] / 800.0 + rng.uniform(0, 6, r)[None, :])).astype(
        np.float32)
    data = np.einsum("pcm,tm->pct", modes, w).astype(np.float32)
    torch.cuda.init()
    snapshot_pod(times[:4], data[:1000, :, :4], 2)  # load the library, warm the context

    def numpy_pod():
        X = data.reshape(-1, t)
        lam, vec = np.linalg.eigh(X.T @ X)
        keep = np.argsort(lam)[::-1][:r]
        phi = X @ (vec[:, keep] / np.sqrt(lam[keep]))
        return phi.reshape(P, 3, r), X.T @ phi

    out = {}
    for name, fn in (("cuda", lambda: snapshot_pod(times, data, r)), ("numpy", numpy_pod)):
        ts = []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            m, wt = fn()
            ts.append(time.perf_counter() - t0)
        out[name] = {"s": statistics.median(ts), "modes": m}
    errs = []
    for m in range(r):
        a, b = out["numpy"]["modes"][..., m], out["cuda"]["modes"][..., m]
        sgn = np.sign(np.vdot(a.ravel(), b.ravel()))
        errs.append(float(np.linalg.norm(a - sgn * b) / np.linalg.norm(a)))
    return {"metric": "POD construction time (method of snapshots, rank 10)", "value": out["cuda"]["s"],
            "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": 1, "ms_per_step": out["cuda"]["s"] * 1e3,
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




def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spawn(n: int) -> int:
    """Re-runs this command as n ranks (one process per GPU) through
    torch.distributed.run, when it was started without a launcher."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(Path(__file__).resolve())]
    cmd += sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="default workload: skip the other configurations' keys")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-step-seconds", type=float, default=3.0)
    ap.add_argument("--f32-steps", type=int, default=5, help="batching: timed steps of the FP32 form")
    ap.add_argument("--tuning", default=None, help="batching: split_nodes/kz_cap instead of the autotuner")
    ap.add_argument("--workload", default="batching",
                    choices=["batching", "plain", "phase_contrast", "precision", "serving", "sequence", "pod",
                             "recon", "node_partition"])
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--slots", type=int, default=16)
    ap.add_argument("--full-sizes", action="store_true", help="serving: add two requests at full sizes")
    ap.add_argument("--spokes", type=int, default=4096)
    ap.add_argument("--check-samples", type=int, default=256)
    ap.add_argument("--phantoms", type=int, default=BATCH_PHANTOMS)
    ap.add_argument("--dummies", type=int, default=80, help="sequence workload: steady-state blocks")
    ap.add_argument("--frames", type=int, default=20, help="sequence workload: stored imaging blocks")
    ap.add_argument("--nodes", type=int, default=N_NODES,
                    help="mesh size (smaller cases of the same workload for profiling)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(_spawn(args.gpus))
    if args.impl == "reference":
        res = run_reference(args)
    elif args.workload == "batching":
        res = run_batching(args)
    elif args.workload == "node_partition":
        res = run_node_partition(args)
    else:
        fn = {"plain": run_plain, "phase_contrast": run_phase_contrast, "precision": run_precision,
              "serving": run_serving, "sequence": run_sequence, "pod": run_pod_build, "recon": run_recon}[args.workload]
        res = fn(args)
        if args.workload in ("plain", "phase_contrast", "precision", "serving"):
            res = dict(res, unit="node*k-sample/s", n_gpus=1, higher_is_better=True, scaling="weak",
                       vs_baseline=None, dtype="bf16x3", data="synthetic",
                       config={"workload": res.get("workload")})
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
