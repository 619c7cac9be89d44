"""Device-level entry points: torch CUDA tensors in, torch CUDA tensors out.

These wrap the C ABI (include/feelmri_b200.h) with PyTorch only as the
allocator of device buffers and the provider of the current stream.  The
drop-in shims (BlochSimulator, MRI, Assemble, POD) convert numpy inputs with
the reference's pybind11 rules and call into here.  No function here computes
on the CPU; without a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from ._motion import LoweredMotion

_ws_cache: dict[tuple[int, int], torch.Tensor] = {}


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("feelmri_b200 runs on a CUDA device (B200, sm_100a); none is available and there "
                           "is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def _index(device: torch.device) -> int:
    return device.index if device.index is not None else torch.cuda.current_device()


def ctx_for(device: torch.device) -> int:
    """Library context of `device` bound to torch's current stream there."""
    stream = torch.cuda.current_stream(device)
    return L.bind_stream(_index(device), stream.cuda_stream)


def workspace(device: torch.device, nbytes: int) -> torch.Tensor:
    """A scratch buffer of at least nbytes, cached per (device, stream).  Work
    on one stream is ordered, so reusing the buffer there is safe."""
    stream = torch.cuda.current_stream(device)
    key = (_index(device), stream.cuda_stream)
    buf = _ws_cache.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=device)
        _ws_cache[key] = buf
    return buf


def release_workspaces() -> None:
    _ws_cache.clear()


_NP_OF = {torch.float32: np.float32, torch.float64: np.float64, torch.int32: np.int32,
          torch.complex64: np.complex64, torch.complex128: np.complex128}
_staging: dict = {}
_staging_lock = None
_copy_pool = None


def upload_many(items, device: torch.device) -> list:
    """Host arrays -> device tensors in one transfer: each (array, torch dtype)
    is converted as `torch.from_numpy(a).to(dtype)` would, copied into one
    pinned staging buffer (on several threads; numpy releases the GIL for
    large copies) and sent with a single host-to-device copy on the current
    stream.  The staging buffer is reused once the previous transfer from it
    has completed (calls from several threads take turns).  Returns the
    tensors (views of one device allocation)."""
    global _staging_lock
    if _staging_lock is None:
        import threading
        _staging_lock = threading.Lock()
    with _staging_lock:
        return _upload_many(items, device)


_COPY_CHUNK = 8 << 20  # bytes of one staging copy task


def _upload_many(items, device: torch.device) -> list:
    global _copy_pool
    arrays, dtypes, offs, total = [], [], [], 0
    for a, dt in items:
        # the conversion to the device dtype happens in the staging copy
        # (np.copyto rounds as astype does), on the copy threads
        arr = np.asarray(a)
        if not arr.flags.c_contiguous:
            arr = np.ascontiguousarray(arr)
        npdt = np.dtype(_NP_OF[dt])
        arrays.append(arr)
        dtypes.append(npdt)
        offs.append(total)
        total += (arr.size * npdt.itemsize + 255) & ~255
    key = _index(device)
    st = _staging.get(key)
    if st is None or st[0].numel() < total:
        st = (torch.empty(max(total, 1 << 20), dtype=torch.uint8, pin_memory=True), None)
    buf, ev = st
    if ev is not None:
        ev.synchronize()  # the last transfer out of this buffer is done
    host = buf.numpy()

    # copy tasks: whole small arrays, large ones in chunks of elements
    tasks = []
    for i, (arr, npdt) in enumerate(zip(arrays, dtypes)):
        n = arr.size
        if n == 0:
            continue
        step = max(1, _COPY_CHUNK // npdt.itemsize)
        for e0 in range(0, n, step):
            tasks.append((i, e0, min(n, e0 + step)))

    def put(task):
        i, e0, e1 = task
        arr, npdt = arrays[i], dtypes[i]
        dst = host[offs[i]:offs[i] + arr.size * npdt.itemsize].view(npdt)
        np.copyto(dst[e0:e1], arr.reshape(-1)[e0:e1], casting="unsafe")
    if len(tasks) > 1 and total >= (2 << 20):
        if _copy_pool is None:
            from concurrent.futures import ThreadPoolExecutor
            _copy_pool = ThreadPoolExecutor(max_workers=8)
        list(_copy_pool.map(put, tasks))
    else:
        for t in tasks:
            put(t)
    dev_buf = torch.empty(max(total, 1), dtype=torch.uint8, device=device)
    dev_buf.copy_(buf[:max(total, 1)], non_blocking=True)
    ev = torch.cuda.Event()
    ev.record(torch.cuda.current_stream(device))
    _staging[key] = (buf, ev)
    out = []
    for (a, dt), arr, npdt, o in zip(items, arrays, dtypes, offs):
        out.append(dev_buf[o:o + arr.size * npdt.itemsize].view(dt).reshape(arr.shape))
    return out


PINNED_RESULT_MAX = 256 << 20


def to_host(*tensors: torch.Tensor):
    """Device results as numpy arrays through pinned staging: the copies are
    queued on the current stream and waited for once.  The arrays keep their
    pinned buffers (torch's caching host allocator takes them back when the
    arrays die); results above PINNED_RESULT_MAX bytes in total are copied to
    pageable memory instead, so that held results do not pin large amounts of
    host memory."""
    if sum(t.numel() * t.element_size() for t in tensors) > PINNED_RESULT_MAX:
        out = [t.cpu().numpy() for t in tensors]
    else:
        staged = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in tensors]
        for h, t in zip(staged, tensors):
            h.copy_(t, non_blocking=True)
        torch.cuda.current_stream(tensors[0].device).synchronize()
        out = [h.numpy() for h in staged]
    return out[0] if len(out) == 1 else tuple(out)


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _check_dev(name: str, t: torch.Tensor, dtype: torch.dtype, shape: tuple, device: torch.device):
    if t.device != device:
        raise ValueError(f"{name} is on {t.device}, expected {device}")
    if t.dtype != dtype:
        raise TypeError(f"{name} has dtype {t.dtype}, expected {dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


# ---------------------------------------------------------------- POD GEMV --

def tensordot_modes_weights(modes: torch.Tensor, weights: torch.Tensor, out: torch.Tensor | None = None):
    """out[p, c] = sum_m modes[p, c, m] * weights[m]  (POD.cpp:5-38)."""
    dev = modes.device
    P, Cc, M = modes.shape
    if out is None:
        out = torch.empty((P, Cc), dtype=modes.dtype, device=dev)
    _check_dev("weights", weights, modes.dtype, (M,), dev)
    fn = L.lib().fm_pod_tensordot_f32 if modes.dtype == torch.float32 else L.lib().fm_pod_tensordot_f64
    L.check(fn(ctx_for(dev), modes.data_ptr(), weights.data_ptr(), P, Cc, M, out.data_ptr()))
    return out


def _pod_ws(rows: int, t: int, r: int, dev) -> torch.Tensor:
    nbytes = C.c_size_t()
    L.check(L.lib().fm_pod_build_workspace_size(rows, t, r, C.byref(nbytes)))
    return workspace(dev, nbytes.value)


def pod_gram(X: torch.Tensor) -> torch.Tensor:
    """X^T X (t x t, float64) of a (rows, t) float32/float64 snapshot matrix."""
    if X.dim() != 2 or X.dtype not in (torch.float32, torch.float64) or not X.is_contiguous():
        raise ValueError("pod_gram: X must be a contiguous (rows, t) float32/float64 tensor")
    rows, t = X.shape
    out = torch.empty((t, t), dtype=torch.float64, device=X.device)
    ws = _pod_ws(rows, t, 0, X.device)
    fn = L.lib().fm_pod_gram_f32 if X.dtype == torch.float32 else L.lib().fm_pod_gram_f64
    L.check(fn(ctx_for(X.device), X.data_ptr(), rows, t, out.data_ptr(), ws.data_ptr(), ws.numel()))
    return out


def pod_project(X: torch.Tensor, E: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """phi = X E (rows x r, X's type) and weights = X^T phi (t x r, float64)."""
    rows, t = X.shape
    if E.dtype != torch.float64 or E.shape[0] != t or E.dim() != 2 or not E.is_contiguous():
        raise ValueError("pod_project: E must be a contiguous (t, r) float64 tensor")
    r = E.shape[1]
    phi = torch.empty((rows, r), dtype=X.dtype, device=X.device)
    weights = torch.empty((t, r), dtype=torch.float64, device=X.device)
    ws = _pod_ws(rows, t, r, X.device)
    fn = L.lib().fm_pod_project_f32 if X.dtype == torch.float32 else L.lib().fm_pod_project_f64
    L.check(fn(ctx_for(X.device), X.data_ptr(), rows, t, E.data_ptr(), r, phi.data_ptr(), weights.data_ptr(),
               ws.data_ptr(), ws.numel()))
    return phi, weights


def motion_eval(motion: LoweredMotion, n_nodes: int, times, device: torch.device) -> torch.Tensor:
    """Displacements (len(times), N, 3) of a lowered motion at host times."""
    times = np.ascontiguousarray(times, dtype=np.float64)
    out = torch.empty((len(times), n_nodes, 3), dtype=torch.float32, device=device)
    nbytes = C.c_size_t()
    L.check(L.lib().fm_motion_eval_workspace_size(C.byref(motion.struct), n_nodes, len(times), C.byref(nbytes)))
    ws = workspace(device, nbytes.value)
    L.check(L.lib().fm_motion_eval(ctx_for(device), C.byref(motion.struct), n_nodes,
                                   times.ctypes.data_as(C.c_void_p), len(times), out.data_ptr(),
                                   ws.data_ptr(), ws.numel()))
    return out


# ------------------------------------------------------------ Bloch sweep --

@dataclass
class BlochInputs:
    """Device-resident inputs of one solve_mri call (all float32/complex64)."""
    r0: torch.Tensor        # (N, 3)
    T1: torch.Tensor        # (N,)
    T2: torch.Tensor        # (N,)
    delta_B: torch.Tensor   # (N,)
    M0: float
    gamma: float
    rf: torch.Tensor        # (n_t,) complex64
    G: torch.Tensor         # (n_t, 3)
    dt: torch.Tensor        # (n_t,)
    Mxy0: torch.Tensor      # (N,) complex64
    Mz0: torch.Tensor       # (N,)


def bloch_solve(inp: BlochInputs, motion: LoweredMotion, history: bool = True,
                Mxy_final: torch.Tensor | None = None, Mz_final: torch.Tensor | None = None,
                Mxy_carry: torch.Tensor | None = None, allocate_final: bool = True):
    """Runs the fused Bloch sweep.  history=True returns the (N, n_t)
    column-major histories (as (n_t, N) row-major tensors); otherwise the
    final state is written to Mxy_final / Mz_final (allocated when None and
    allocate_final) and 0 * final Mxy to Mxy_carry when given.  The output
    buffers may alias Mxy0 / Mz0 (each node is read before it is written)."""
    dev = inp.r0.device
    N = inp.r0.shape[0]
    n_t = inp.rf.shape[0]
    _check_dev("r0", inp.r0, torch.float32, (N, 3), dev)
    for name in ("T1", "T2", "delta_B", "Mz0"):
        _check_dev(name, getattr(inp, name), torch.float32, (N,), dev)
    _check_dev("Mxy0", inp.Mxy0, torch.complex64, (N,), dev)
    _check_dev("rf", inp.rf, torch.complex64, (n_t,), dev)
    _check_dev("G", inp.G, torch.float32, (n_t, 3), dev)
    _check_dev("dt", inp.dt, torch.float32, (n_t,), dev)
    a = L.BlochArgs()
    a.n_pos, a.n_time = N, n_t
    a.r0, a.T1, a.T2, a.delta_B = (_ptr(inp.r0), _ptr(inp.T1), _ptr(inp.T2), _ptr(inp.delta_B))
    a.M0, a.gamma = float(np.float32(inp.M0)), float(np.float32(inp.gamma))
    a.rf, a.G, a.dt = _ptr(inp.rf), _ptr(inp.G), _ptr(inp.dt)
    a.Mxy0, a.Mz0 = _ptr(inp.Mxy0), _ptr(inp.Mz0)
    a.motion = C.pointer(motion.struct)
    hist = None
    if history:
        Mxy_h = torch.empty((n_t, N), dtype=torch.complex64, device=dev)
        Mz_h = torch.empty((n_t, N), dtype=torch.float32, device=dev)
        a.Mxy_hist, a.Mz_hist = Mxy_h.data_ptr(), Mz_h.data_ptr()
        hist = (Mxy_h, Mz_h)
    if Mxy_final is None and not history and allocate_final:
        Mxy_final = torch.empty((N,), dtype=torch.complex64, device=dev)
    if Mz_final is None and not history and allocate_final:
        Mz_final = torch.empty((N,), dtype=torch.float32, device=dev)
    for name, buf, dt in (("Mz_final", Mz_final, torch.float32), ("Mxy_carry", Mxy_carry, torch.complex64)):
        if buf is not None:
            _check_dev(name, buf, dt, (N,), dev)
    if Mxy_final is not None:
        # a 1-D view with any positive stride, e.g. one column of an (N, V) matrix
        if Mxy_final.device != dev or Mxy_final.dtype != torch.complex64 or tuple(Mxy_final.shape) != (N,):
            raise ValueError("Mxy_final must be a complex64 (N,) tensor on the solve's device")
        if Mxy_final.stride(0) < 1:
            raise ValueError("Mxy_final must have a positive stride")
        a.final_stride = Mxy_final.stride(0)
    a.Mxy_final, a.Mz_final, a.Mxy_carry = _ptr(Mxy_final), _ptr(Mz_final), _ptr(Mxy_carry)
    nbytes = C.c_size_t()
    L.check(L.lib().fm_bloch_workspace_size(C.byref(a), C.byref(nbytes)))
    ws = workspace(dev, nbytes.value)
    L.check(L.lib().fm_bloch_solve_f32(ctx_for(dev), C.byref(a), ws.data_ptr(), ws.numel()))
    if history:
        return hist
    return Mxy_final, Mz_final


@dataclass
class SequenceBlock:
    """One block of a device-side block sequence (fm_bloch_sequence_f32)."""
    n_time: int
    empty: bool = False
    store: int = -1                    # row of the stored final states, or -1
    timeshifts: tuple = ()             # ((value, FM_NUM_* kind), ...) per motion term


def bloch_sequence(r0: torch.Tensor, T1: torch.Tensor, T2: torch.Tensor, delta_B: torch.Tensor, M0: float,
                   gamma: float, blocks: list[SequenceBlock], rf: torch.Tensor, G: torch.Tensor, dt: torch.Tensor,
                   Mxy0: torch.Tensor, Mz0: torch.Tensor, motion: LoweredMotion, Mxy_out: torch.Tensor,
                   Mz_out: torch.Tensor, Mxy_carry: torch.Tensor | None = None,
                   Mz_carry: torch.Tensor | None = None) -> None:
    """Runs a whole block sequence in one sweep: rf / G / dt hold the blocks'
    samples concatenated in block order; block i's final state goes to row
    blocks[i].store of Mxy_out / Mz_out when that is >= 0; the state carried
    past the last block goes to Mxy_carry / Mz_carry (which may alias Mxy0 /
    Mz0).  motion is NONE or TERMS (the per-block timeshifts replace its
    terms')."""
    dev = r0.device
    N = r0.shape[0]
    S = rf.shape[0]
    _check_dev("r0", r0, torch.float32, (N, 3), dev)
    for name, t in (("T1", T1), ("T2", T2), ("delta_B", delta_B), ("Mz0", Mz0)):
        _check_dev(name, t, torch.float32, (N,), dev)
    _check_dev("Mxy0", Mxy0, torch.complex64, (N,), dev)
    _check_dev("rf", rf, torch.complex64, (S,), dev)
    _check_dev("G", G, torch.float32, (S, 3), dev)
    _check_dev("dt", dt, torch.float32, (S,), dev)
    n_store = Mxy_out.shape[0]
    _check_dev("Mxy_out", Mxy_out, torch.complex64, (n_store, N), dev)
    _check_dev("Mz_out", Mz_out, torch.float32, (n_store, N), dev)
    if Mxy_carry is not None:
        _check_dev("Mxy_carry", Mxy_carry, torch.complex64, (N,), dev)
    if Mz_carry is not None:
        _check_dev("Mz_carry", Mz_carry, torch.float32, (N,), dev)
    table = (L.BlochBlock * max(len(blocks), 1))()
    off = 0
    for i, b in enumerate(blocks):
        e = table[i]
        e.offset, e.n_time, e.empty, e.store = off, int(b.n_time), int(bool(b.empty)), int(b.store)
        for k, (v, kind) in enumerate(b.timeshifts):
            e.timeshift[k], e.timeshift_kind[k] = float(v), int(kind)
        off += int(b.n_time)
    a = L.BlochSequenceArgs()
    a.n_pos = N
    a.r0, a.T1, a.T2, a.delta_B = _ptr(r0), _ptr(T1), _ptr(T2), _ptr(delta_B)
    a.M0, a.gamma = float(np.float32(M0)), float(np.float32(gamma))
    a.n_blocks, a.blocks, a.n_samples = len(blocks), table, S
    a.rf, a.G, a.dt = _ptr(rf), _ptr(G), _ptr(dt)
    a.Mxy0, a.Mz0 = _ptr(Mxy0), _ptr(Mz0)
    a.motion = C.pointer(motion.struct)
    a.n_store, a.Mxy_out, a.Mz_out = n_store, _ptr(Mxy_out), _ptr(Mz_out)
    a.Mxy_carry, a.Mz_carry = _ptr(Mxy_carry), _ptr(Mz_carry)
    nbytes = C.c_size_t()
    L.check(L.lib().fm_bloch_sequence_workspace_size(C.byref(a), C.byref(nbytes)))
    ws = workspace(dev, nbytes.value)
    L.check(L.lib().fm_bloch_sequence_f32(ctx_for(dev), C.byref(a), ws.data_ptr(), ws.numel()))


# ----------------------------------------------------------------- Signal --

@dataclass
class SparseCSC:
    """A CSC matrix on the device (int32 index arrays)."""
    shape: tuple
    indptr: torch.Tensor
    indices: torch.Tensor
    data: torch.Tensor

    @property
    def nnz(self) -> int:
        return int(self.indices.numel())


@dataclass
class SignalInputs:
    """Device-resident inputs of one Signal call.  Real arrays are float32 for
    the F32 and BF16X3 forms and float64 for the F64 form."""
    M: SparseCSC
    kx: torch.Tensor      # (n_ro, n_lines, n_kz)
    ky: torch.Tensor
    kz: torch.Tensor
    t: torch.Tensor       # (n_ro, n_lines, n_kz)
    r0: torch.Tensor      # (N, 3)
    phi: torch.Tensor     # (N,)
    T2: torch.Tensor      # (N,)
    Mxy: torch.Tensor     # (N, V) complex


PRECISIONS = {"f32": L.FM_PREC_F32, "f64": L.FM_PREC_F64, "bf16x3": L.FM_PREC_BF16X3}


def signal_args(inp: SignalInputs, motion: LoweredMotion, precision: str, out: torch.Tensor) -> L.SignalArgs:
    real = torch.float64 if precision == "f64" else torch.float32
    cplx = torch.complex128 if precision == "f64" else torch.complex64
    dev = inp.r0.device
    N = inp.r0.shape[0]
    V = inp.Mxy.shape[1]
    grid = tuple(inp.kx.shape)
    if len(grid) != 3:
        raise ValueError("k-space arrays must be 3-D (n_ro, n_lines, n_kz)")
    for name in ("kx", "ky", "kz", "t"):
        _check_dev(name, getattr(inp, name), real, grid, dev)
    _check_dev("r0", inp.r0, real, (N, 3), dev)
    _check_dev("phi", inp.phi, real, (N,), dev)
    _check_dev("T2", inp.T2, real, (N,), dev)
    _check_dev("Mxy", inp.Mxy, cplx, (N, V), dev)
    _check_dev("M.data", inp.M.data, real, (inp.M.nnz,), dev)
    _check_dev("out", out, cplx, (*grid, V), dev)
    a = L.SignalArgs()
    a.n_nodes, a.n_vencs = N, V
    a.n_ro, a.n_lines, a.n_kz = grid
    a.m_rows, a.m_cols = inp.M.shape
    a.m_nnz = inp.M.nnz
    a.m_indptr, a.m_indices, a.m_data = _ptr(inp.M.indptr), _ptr(inp.M.indices), _ptr(inp.M.data)
    a.kx, a.ky, a.kz, a.t = _ptr(inp.kx), _ptr(inp.ky), _ptr(inp.kz), _ptr(inp.t)
    a.r0, a.phi, a.T2, a.Mxy = _ptr(inp.r0), _ptr(inp.phi), _ptr(inp.T2), _ptr(inp.Mxy)
    a.motion = C.pointer(motion.struct)
    a.out = out.data_ptr()
    return a


def signal(inp: SignalInputs, motion: LoweredMotion, precision: str = "f32",
           out: torch.Tensor | None = None, sync: bool = True, ws: torch.Tensor | None = None) -> torch.Tensor:
    """k-space (n_ro, n_lines, n_kz, V) of the mass-weighted NUDFT.  With
    sync=False the work is only queued on the current stream (no host wait);
    call signal_status with the same inputs and workspace to collect errors."""
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    dev = inp.r0.device
    cplx = torch.complex128 if precision == "f64" else torch.complex64
    if out is None:
        out = torch.empty((*inp.kx.shape, inp.Mxy.shape[1]), dtype=cplx, device=dev)
    a = signal_args(inp, motion, precision, out)
    if ws is None:
        ws = workspace(dev, signal_workspace_bytes(a, precision))
    fn = L.lib().fm_signal if sync else L.lib().fm_signal_enqueue
    L.check(fn(ctx_for(dev), C.byref(a), PRECISIONS[precision], ws.data_ptr(), ws.numel()))
    return out


@dataclass(frozen=True)
class Tuning:
    """Work-unit shape of the batched tensor-core Signal (fm_tc_tuning):
    nodes per unit (0: spread each problem over the SMs) and the most kz
    values per tile (0: up to 64)."""
    split_nodes: int = 0
    kz_cap: int = 0

    def struct(self) -> L.TcTuning:
        t = L.TcTuning()
        t.split_nodes, t.kz_cap = int(self.split_nodes), int(self.kz_cap)
        return t


class SignalBatch:
    """n split-BF16 Signal problems contracted by one persistent tensor-core
    launch.  Holds the argument array, the lowered motions and the workspace,
    so a batch can be enqueued repeatedly (for instance inside a CUDA graph
    capture) with the same buffers."""

    def __init__(self, problems: list[tuple[SignalInputs, LoweredMotion, torch.Tensor]],
                 tuning: Tuning | None = None):
        if not problems:
            raise ValueError("empty batch")
        self.dev = problems[0][0].r0.device
        self.problems = problems  # keeps the motion descriptors alive
        self.tuning = tuning or Tuning()
        self._tune = self.tuning.struct()
        self.args = (L.SignalArgs * len(problems))()
        for i, (inp, motion, out) in enumerate(problems):
            if inp.r0.device != self.dev:
                raise ValueError("all problems of a batch must be on one device")
            self.args[i] = signal_args(inp, motion, "bf16x3", out)
        nbytes = C.c_size_t()
        L.check(L.lib().fm_signal_batch_workspace_size(self.args, len(problems), C.byref(nbytes)))
        self.ws = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=self.dev)

    @property
    def outs(self) -> list[torch.Tensor]:
        return [o for _, _, o in self.problems]

    def enqueue(self) -> None:
        """Queues the batch on the current stream (no host wait)."""
        L.check(L.lib().fm_signal_batch_enqueue(ctx_for(self.dev), self.args, len(self.problems),
                                                C.byref(self._tune), self.ws.data_ptr(), self.ws.numel()))

    def status(self) -> None:
        """Waits for the stream and raises the errors the device work found."""
        L.check(L.lib().fm_signal_batch_status(ctx_for(self.dev), self.args, len(self.problems),
                                               self.ws.data_ptr(), self.ws.numel()))

    def run(self) -> list[torch.Tensor]:
        self.enqueue()
        self.status()
        return self.outs


def signal_batch(problems: list[tuple[SignalInputs, LoweredMotion, torch.Tensor | None]],
                 tuning: Tuning | None = None) -> list[torch.Tensor]:
    """Split-BF16 k-spaces of several problems (each (inputs, motion, out or
    None)) from one persistent tensor-core launch."""
    full = []
    for inp, motion, out in problems:
        if out is None:
            out = torch.empty((*inp.kx.shape, inp.Mxy.shape[1]), dtype=torch.complex64, device=inp.r0.device)
        full.append((inp, motion, out))
    return SignalBatch(full, tuning).run()


def signal_workspace_bytes(a: L.SignalArgs, precision: str) -> int:
    nbytes = C.c_size_t()
    L.check(L.lib().fm_signal_workspace_size(C.byref(a), PRECISIONS[precision], C.byref(nbytes)))
    return nbytes.value


def signal_status(inp: SignalInputs, motion: LoweredMotion, precision: str, out: torch.Tensor,
                  ws: torch.Tensor) -> None:
    """Waits for a queued signal() and raises the errors its device work found."""
    a = signal_args(inp, motion, precision, out)
    L.check(L.lib().fm_signal_status(ctx_for(inp.r0.device), C.byref(a), PRECISIONS[precision], ws.data_ptr(),
                                     ws.numel()))


def coil_expand(m: torch.Tensor, sens: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """(N, C) complex64 columns m[n] * sens[n, c] (receive coils)."""
    dev = m.device
    N, Cc = sens.shape
    _check_dev("m", m, torch.complex64, (N,), dev)
    _check_dev("sens", sens, torch.complex64, (N, Cc), dev)
    if out is None:
        out = torch.empty((N, Cc), dtype=torch.complex64, device=dev)
    L.check(L.lib().fm_coil_expand(ctx_for(dev), m.data_ptr(), sens.data_ptr(), N, Cc, out.data_ptr()))
    return out


def count_time_runs(t: np.ndarray) -> int:
    t = np.ascontiguousarray(t).reshape(-1)
    return int(L.lib().fm_signal_count_time_runs(t.ctypes.data_as(C.c_void_p), t.size,
                                                 1 if t.dtype == np.float64 else 0))


# ------------------------------------------------------------------- Mass --

def _mass_args(elems: torch.Tensor, nodes: torch.Tensor, qweights: torch.Tensor, tab: torch.Tensor) -> L.MassArgs:
    dev = nodes.device
    E, nb = elems.shape
    N = nodes.shape[0]
    Q = qweights.shape[0]
    _check_dev("elems", elems, torch.int32, (E, nb), dev)
    _check_dev("nodes", nodes, nodes.dtype, (N, 3), dev)
    _check_dev("qweights", qweights, nodes.dtype, (Q,), dev)
    _check_dev("tabulated", tab, nodes.dtype, (Q, 4, nb), dev)
    a = L.MassArgs()
    a.n_elems, a.nodes_per_elem = E, nb
    a.elems = _ptr(elems)
    a.n_nodes = N
    a.nodes = _ptr(nodes)
    a.n_qpoints = Q
    a.qweights = _ptr(qweights)
    a.tabulated = _ptr(tab)
    return a


def mass_assemble(elems, nodes, qweights, tab):
    """CSC (indptr, indices, data) of the assembled mass matrix."""
    dev = nodes.device
    is_double = 1 if nodes.dtype == torch.float64 else 0
    a = _mass_args(elems, nodes, qweights, tab)
    nbytes = C.c_size_t()
    L.check(L.lib().fm_mass_workspace_size(C.byref(a), is_double, C.byref(nbytes)))
    ws = workspace(dev, nbytes.value)
    nnz = C.c_int64()
    N = nodes.shape[0]
    indptr = torch.empty((N + 1,), dtype=torch.int32, device=dev)
    ctx = ctx_for(dev)
    L.check(L.lib().fm_mass_assemble(ctx, C.byref(a), is_double, C.byref(nnz), indptr.data_ptr(), None, None, 0,
                                     ws.data_ptr(), ws.numel()))
    indices = torch.empty((nnz.value,), dtype=torch.int32, device=dev)
    data = torch.empty((nnz.value,), dtype=nodes.dtype, device=dev)
    L.check(L.lib().fm_mass_assemble(ctx, C.byref(a), is_double, C.byref(nnz), indptr.data_ptr(),
                                     indices.data_ptr(), data.data_ptr(), nnz.value, ws.data_ptr(), ws.numel()))
    return indptr, indices, data


def mass_lumped(elems, nodes, qweights, tab) -> torch.Tensor:
    """Row sums of the assembled mass matrix (FEMPhantom.mass_matrix(lumped=True))."""
    dev = nodes.device
    is_double = 1 if nodes.dtype == torch.float64 else 0
    a = _mass_args(elems, nodes, qweights, tab)
    nbytes = C.c_size_t()
    L.check(L.lib().fm_mass_workspace_size(C.byref(a), is_double, C.byref(nbytes)))
    ws = workspace(dev, nbytes.value)
    out = torch.empty((nodes.shape[0],), dtype=nodes.dtype, device=dev)
    L.check(L.lib().fm_mass_lumped(ctx_for(dev), C.byref(a), is_double, out.data_ptr(), ws.data_ptr(),
                                   ws.numel()))
    return out
