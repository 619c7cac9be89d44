"""Image-domain reconstruction on the GPU with exact NUDFT operators.

The reference reconstructs with pynufft's gridding NUFFT
(python/feelmri/Recon.py:151-290, `reconstruct_nufft`: an adjoint after
Pipe-Menon, radial-ramp or readout-speed density compensation).  This module
gives the same operations with the exact non-uniform DFT instead of a gridding
approximation, built on the Signal contraction (fm_signal), read the other
way round:

* forward, image -> k-space:  K[s, c] = sum_n I[n, c] exp(-2 pi i k_s . x_n),
  which is Signal with the voxel centres as nodes;
* adjoint, k-space -> image:  I[n, c] = sum_s w_s K[s, c] exp(+2 pi i k_s . x_n),
  which is Signal with the roles swapped: the k-space samples act as the
  nodes (their k vectors as positions, the density weights as the lumped
  mass) and the voxel centres, negated, as the sample points.

The voxel grid is Cartesian, so in the adjoint every x-slice of the image is a
(y x z) slab with k = kp + kq exactly: the split-BF16 tensor-core form factors
it whatever the trajectory (radial, spiral, Cartesian).  Phases use the
Signal's float-rounded pi (cpp/feelmri/MRI.h:13); decay and off-resonance are
switched off (T2 = inf, phi = 0).

Conventions (physical units, as the simulator's): k in 1/m; the image has
shape (Nx, Ny, Nz) over a field of view (FOVx, FOVy, FOVz) in m, with voxel
centres x_d = n_d * FOV_d / N_d for n_d = -N_d // 2 .. N_d - N_d // 2 - 1
(the DFT-centred grid).  pynufft's scaling and deapodisation are not
reproduced: these are the exact sums above.
"""
from __future__ import annotations

import numpy as np
import torch

from . import ops
from ._motion import lower

__all__ = ["grid_points", "nudft_forward", "nudft_adjoint", "dcf_pipe_menon", "dcf_path_jacobian",
           "reconstruct_nudft", "cartesian_recon", "CartesianRecon"]


def grid_points(img_shape, fov) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Voxel-centre coordinates (X, Y, Z), each shaped img_shape, float32 metres."""
    shape = tuple(int(n) for n in img_shape)
    if len(shape) != 3 or len(fov) != 3:
        raise ValueError("img_shape and fov must have three entries (use 1 for a 2-D image)")
    axes = [(np.arange(n) - n // 2).astype(np.float64) * (float(f) / n) for n, f in zip(shape, fov)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    return X.astype(np.float32), Y.astype(np.float32), Z.astype(np.float32)


def _up(a, dtype, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dtype)


def _diag_csc(w: np.ndarray, dev) -> ops.SparseCSC:
    n = w.shape[0]
    idx = torch.arange(n + 1, dtype=torch.int32, device=dev)
    return ops.SparseCSC((n, n), idx, idx[:n], _up(w, torch.float32, dev))


def _check_precision(precision: str):
    if precision not in ("bf16x3", "f32"):
        raise ValueError(f"precision must be 'bf16x3' or 'f32'; got {precision!r}")


def nudft_adjoint(kdata, kx, ky, kz, img_shape, fov, dcw=None, precision: str = "bf16x3") -> np.ndarray:
    """I[n, c] = sum_s dcw_s kdata[s, c] exp(+2 pi i k_s . x_n) on the voxel
    grid; kdata (S, C) or (..., C) complex with kx, ky, kz of S samples (any
    shape) in 1/m.  Returns (Nx, Ny, Nz, C) complex64."""
    _check_precision(precision)
    dev = ops.require_cuda()
    k = np.stack([np.asarray(a, np.float32).reshape(-1) for a in (kx, ky, kz)], axis=1)
    S = k.shape[0]
    K = np.asarray(kdata).reshape(S, -1).astype(np.complex64)
    w = np.ones(S, np.float32) if dcw is None else np.asarray(dcw, np.float32).reshape(-1)
    if w.shape[0] != S:
        raise ValueError(f"dcw has {w.shape[0]} weights for {S} samples")
    X, Y, Z = grid_points(img_shape, fov)
    # one run per x-slice: every slice is a (y, z) slab that factors exactly
    t = np.broadcast_to(np.arange(X.shape[0], dtype=np.float32)[:, None, None], X.shape)
    inp = ops.SignalInputs(M=_diag_csc(w, dev), kx=_up(-X, torch.float32, dev), ky=_up(-Y, torch.float32, dev),
                           kz=_up(-Z, torch.float32, dev), t=_up(t, torch.float32, dev), r0=_up(k, torch.float32, dev),
                           phi=torch.zeros(S, dtype=torch.float32, device=dev),
                           T2=torch.full((S,), float("inf"), dtype=torch.float32, device=dev),
                           Mxy=_up(K, torch.complex64, dev))
    return ops.to_host(ops.signal(inp, lower(None, S, dev), precision))


def nudft_forward(image, kx, ky, kz, fov, t=None, precision: str = "bf16x3") -> np.ndarray:
    """K[s, c] = sum_n image[n, c] exp(-2 pi i k_s . x_n) for an (Nx, Ny, Nz, C)
    image; kx, ky, kz (R, L, S) in 1/m (a Cartesian stack factors when each
    readout index is one (line, kz) slab: pass the readout times as t, or the
    readout index is used).  Returns (R, L, S, C) complex64."""
    _check_precision(precision)
    dev = ops.require_cuda()
    img = np.asarray(image)
    if img.ndim == 3:
        img = img[..., None]
    X, Y, Z = grid_points(img.shape[:3], fov)
    N = X.size
    kx3, ky3, kz3 = (np.asarray(a, np.float32) for a in (kx, ky, kz))
    if kx3.ndim != 3 or kx3.shape != ky3.shape or kx3.shape != kz3.shape:
        raise ValueError("kx, ky, kz must share one (R, L, S) shape")
    if t is None:
        t = np.broadcast_to(np.arange(kx3.shape[0], dtype=np.float32)[:, None, None], kx3.shape)
    r0 = np.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)], axis=1)
    inp = ops.SignalInputs(M=_diag_csc(np.ones(N, np.float32), dev), kx=_up(kx3, torch.float32, dev),
                           ky=_up(ky3, torch.float32, dev), kz=_up(kz3, torch.float32, dev),
                           t=_up(np.asarray(t, np.float32), torch.float32, dev), r0=_up(r0, torch.float32, dev),
                           phi=torch.zeros(N, dtype=torch.float32, device=dev),
                           T2=torch.full((N,), float("inf"), dtype=torch.float32, device=dev),
                           Mxy=_up(img.reshape(N, -1).astype(np.complex64), torch.complex64, dev))
    return ops.to_host(ops.signal(inp, lower(None, N, dev), precision))


def dcf_pipe_menon(kx, ky, kz, img_shape, fov, n_iter: int = 20, eps: float = 1e-8, window_sigma=None,
                   precision: str = "bf16x3") -> np.ndarray:
    """Pipe-Menon iterative density compensation (Recon.py:95-106),
    w <- w / Re(A C A^H w), normalised to mean 1.

    The reference's A A^H is pynufft's gridding operator pair, whose implied
    k-space kernel is the (positive) interpolation kernel.  With exact
    operators A A^H convolves with the grid's Dirichlet kernel, which has
    negative lobes, and the iteration need not stay positive.  C is therefore
    an image-space Gaussian window (standard deviations window_sigma, default
    FOV / (2 pi) per axis): A C A^H then convolves with a positive Gaussian of
    about one k-space grid step, and the weights stay positive.  Choose the
    grid so that it covers the trajectory (N_d >= 2 kmax_d FOV_d), as for the
    reconstruction itself.  Returns the weights of kx.size samples (C order)."""
    kx3 = np.asarray(kx, np.float32)
    shape3 = kx3.shape if kx3.ndim == 3 else (kx3.size, 1, 1)
    kx3, ky3, kz3 = (np.asarray(a, np.float32).reshape(shape3) for a in (kx, ky, kz))
    sig = [f / (2 * np.pi) for f in fov] if window_sigma is None else list(window_sigma)
    X, Y, Z = grid_points(img_shape, fov)
    window = np.exp(-0.5 * ((X / sig[0]) ** 2 + (Y / sig[1]) ** 2 + (Z / sig[2]) ** 2)).astype(np.float32)
    w = np.ones(kx3.size, np.float32)
    for _ in range(n_iter):
        img = nudft_adjoint(w[:, None], kx3, ky3, kz3, img_shape, fov, precision=precision)
        g = nudft_forward(img * window[..., None], kx3, ky3, kz3, fov, precision=precision).reshape(-1)
        w = (w / (np.real(g) + eps)).astype(np.float32)
    return (w / (w.mean() + eps)).astype(np.float32)


def dcf_path_jacobian(kx, ky, kz=None, radial_power: int = 1) -> np.ndarray:
    """Analytic density weights from the geometry of the readout paths.

    Samples along one readout (axis 0 of the (R, L, S) arrays) cover a
    stretch of path of length v_i = |dk/di| (central differences inside the
    readout, one-sided at its ends, np.gradient); paths that fan out from the
    centre (radials, spirals) thin out with the in-plane radius rho, so
    each sample represents an area proportional to v_i * rho_i^radial_power
    (radial_power = 1 for 2-D fans and stacks of them, 2 for 3-D radials,
    0 for parallel lines).  Returned flattened in C order, scaled to mean 1."""
    kx = np.asarray(kx, np.float64)
    ky = np.asarray(ky, np.float64)
    if kx.ndim != 3 or kx.shape != ky.shape:
        raise ValueError(f"kx and ky must be (R, L, S) arrays of one shape, got {kx.shape} and {ky.shape}")
    parts = [kx, ky] if kz is None else [kx, ky, np.asarray(kz, np.float64)]
    if kx.shape[0] < 2:
        speed = np.ones_like(kx)
    else:
        speed = np.sqrt(sum(np.gradient(p, axis=0) ** 2 for p in parts))
    rho = np.hypot(kx, ky) if radial_power != 2 or kz is None else np.sqrt(sum(p ** 2 for p in parts))
    w = speed * rho ** radial_power
    mean = w.mean()
    return (w / mean if mean > 0 else np.ones_like(w)).astype(np.float32).reshape(-1)


def reconstruct_nudft(kdata, ktraj, img_shape, fov, *, dcw=None, auto_dcw: str | None = "pipe-menon",
                      n_iter: int = 20, combine: str | None = None, precision: str = "bf16x3") -> np.ndarray:
    """Image from non-Cartesian k-space with the exact NUDFT adjoint (the task
    of reconstruct_nufft, Recon.py:150-290, which uses pynufft's gridding
    approximation instead).  kdata (R, L, S, C), ktraj = (kx, ky, kz) each
    (R, L, S) in 1/m (kz may be None for 2-D), img_shape (Nx, Ny, Nz), fov in
    m.  Density weights: dcw when given, else auto_dcw: None (no weights),
    'pipe-menon' (dcf_pipe_menon) or 'jacobian' (dcf_path_jacobian).
    Returns (Nx, Ny, Nz) for one channel or combine='rss', else
    (C, Nx, Ny, Nz)."""
    kx, ky, kz = ktraj
    kx = np.asarray(kx, np.float32)
    ky = np.asarray(ky, np.float32)
    kz = np.zeros_like(kx) if kz is None else np.asarray(kz, np.float32)
    if not (kx.shape == ky.shape == kz.shape) or kx.ndim != 3:
        raise ValueError(f"trajectory arrays must all be (R, L, S); got {kx.shape}, {ky.shape}, {kz.shape}")
    kdata = np.asarray(kdata)
    if kdata.ndim != 4 or kdata.shape[:3] != kx.shape:
        raise ValueError(f"k-space data of shape {kdata.shape} does not fit a {kx.shape} trajectory with a "
                         "trailing channel axis")
    n_ch = kdata.shape[3]
    n_samples = kx.size
    if dcw is None and auto_dcw is not None:
        kind = auto_dcw.lower()
        if kind == "pipe-menon":
            dcw = dcf_pipe_menon(kx, ky, kz, img_shape, fov, n_iter=n_iter, precision=precision)
        elif kind == "jacobian":
            dcw = dcf_path_jacobian(kx, ky, None if not np.any(kz) else kz)
        else:
            raise ValueError(f"unknown auto_dcw {auto_dcw!r}: use None, 'pipe-menon' or 'jacobian'")
    if dcw is not None:
        dcw = np.asarray(dcw, np.float32).reshape(-1)
        if dcw.size != n_samples:
            raise ValueError(f"{dcw.size} density weights for {n_samples} samples")
    img = nudft_adjoint(kdata.reshape(n_samples, n_ch), kx, ky, kz, img_shape, fov, dcw=dcw, precision=precision)
    img = np.moveaxis(img, -1, 0)  # (C, Nx, Ny, Nz)
    if n_ch == 1:
        return img[0]
    if combine is None:
        return img
    if combine.lower() == "rss":
        return np.sqrt(np.sum(np.abs(img) ** 2, axis=0)).astype(np.complex64)
    raise ValueError(f"unknown combine {combine!r}: use None or 'rss'")


# ------------------------------------------------------- Cartesian recon --

def _kspace_window(n: int, kind: str, width: float = 0.9, lift: float = 0.3) -> np.ndarray:
    """1-D k-space apodisation of length n.  'Tukey': a Tukey window with
    taper fraction 1 - width, lifted to [lift, 1]; 'Riesz': flat in the
    middle `width` of the axis, falling as 1 - (1 - lift) (d / d0)^2 over
    each end stretch of round((1 - width) n / 2) samples (d the distance
    into the stretch from its inner edge, d0 half the stretch length)."""
    if kind == "Tukey":
        from scipy.signal.windows import tukey
        return tukey(n, alpha=1.0 - width) * (1.0 - lift) + lift
    if kind == "Riesz":
        m = int(np.round((1.0 - width) / 2 * n))
        h = np.ones(n)
        if m > 0:
            d = np.linspace(0.0, m / 2, m)
            edge = 1.0 - (np.abs(d / (m / 2)) ** 2) * (1.0 - lift)
            h[:m] *= edge[::-1]
            h[n - m:] *= edge
        return h
    return np.ones(n)


def cartesian_recon(K, trajectory, filter=None) -> np.ndarray:
    """Image from Cartesian k-space by the inverse FFT on the GPU, with the
    steps of CartesianRecon (python/feelmri/Recon.py:13-90):

    * for a CartesianStack with several lines per shot, lines read in the
      reverse direction (odd positions within their shot) are flipped along
      the readout;
    * axes 0-2 with an even resolution are zero-padded by one sample at the
      end (so that the image is not shifted);
    * the k-space is apodised along the readout and phase axes by a Tukey or
      Riesz window (width 0.9, lift 0.3, as the reference fixes them; any
      other filter type applies none);
    * the centred inverse FFT over axes 0-2 (torch.fft on the device);
    * the image is brought to oversampling x res along the first three axes
      by trilinear interpolation when the shapes differ, then the readout is
      cut to res[0] around its centre.

    K: (n_ro, n_lines, n_kz, ...) complex; trajectory: an object with .res,
    .oversampling_arr and, for line reordering, .lines_per_shot and .shots
    (the reference's CartesianStack attributes).  Returns complex64 of shape
    (res[0], res[1], res[2], ...) (the reference's interpolation differs
    in detail when shapes change: skimage's resize, not available here)."""
    dev = ops.require_cuda()
    kind = (filter or {"type": "Tukey"}).get("type")
    K = np.array(K, dtype=np.complex64, copy=True)
    if K.ndim < 3:
        raise ValueError(f"K must have at least 3 dimensions (readout, lines, kz), got {K.shape}")
    extra = K.shape[3:]
    res = np.asarray(trajectory.res).astype(int)
    lps = int(getattr(trajectory, "lines_per_shot", 1) or 1)
    if lps > 1:
        for shot in getattr(trajectory, "shots", []):
            for pos, line in enumerate(shot):
                if pos % 2 == 1 and line is not None:
                    K[:, line] = K[::-1, line].copy()
    pad = [(0, 1) if res[d] % 2 == 0 else (0, 0) for d in range(3)] + [(0, 0)] * len(extra)
    if any(p != (0, 0) for p in pad):
        K = np.pad(K, pad)
    h = np.outer(_kspace_window(K.shape[0], kind), _kspace_window(K.shape[1], kind)).astype(np.float32)
    t = torch.from_numpy(K).to(dev)
    t = t * torch.from_numpy(h).to(dev).reshape(h.shape + (1,) * (K.ndim - 2))
    dims = (0, 1, 2)
    img = torch.fft.fftshift(torch.fft.ifftn(torch.fft.ifftshift(t, dim=dims), dim=dims), dim=dims)
    target = tuple(int(round(x)) for x in np.asarray(trajectory.oversampling_arr) * res)
    if tuple(img.shape[:3]) != target:
        flat = img.reshape(img.shape[:3] + (-1,)).permute(3, 0, 1, 2)  # (C, X, Y, Z)
        parts = [torch.nn.functional.interpolate(part.unsqueeze(0), size=target, mode="trilinear",
                                                 align_corners=False)[0]
                 for part in (flat.real.contiguous(), flat.imag.contiguous())]
        img = torch.complex(parts[0], parts[1]).permute(1, 2, 3, 0).reshape(target + extra)
    enc, rec = img.shape[0], int(res[0])
    if enc != rec:
        a = (enc - rec) // 2
        img = img[a:a + rec]
    return ops.to_host(img.contiguous())


# the reference's name for the same call
CartesianRecon = cartesian_recon
