"""Seeded synthetic inputs for the simulation hot path.

The reference's example phantoms are not available, so meshes, tissue
parameters, sequences, trajectories and motion are generated here with
numpy.random.default_rng(seed):

* meshes: a structured grid of cubes split into six tetrahedra (Kuhn split),
  keeping the cells whose centroid lies inside the body; nodes are the sorted
  unique used vertices, as FEMPhantom's local numbering (Phantom.py:215-224);
* sequences: hard-pulse spoiled gradient echo (one block per TR, discretised
  at 10 us during RF and coarser in between) and phase-contrast imaging
  blocks with bipolar velocity-encoding lobes;
* trajectories: Cartesian stacks whose sample time depends on the readout
  index (KSpaceTraj.py:180-220), 3-D radial spokes on a Fibonacci sphere and
  stacks of spirals;
* motion: Poiseuille flow as a rank-1 velocity-mode motion and sinusoidal
  mode weights (feelmri_b200.motion.SplineMotion).

Units follow the reference: ms, mT, m, rad/(ms mT), 1/m.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

GAMMA = 42.58e6 * 2 * np.pi * 1e-6  # rad/(ms mT): 267.5 (MRObjects.py:39-40)
GAMMABAR = 42.58e6 * 1e-6           # cycles/(ms mT)


# ------------------------------------------------------------------ meshes --

@dataclass
class Mesh:
    nodes: np.ndarray   # (N, 3) float64
    elems: np.ndarray   # (E, 4) int32

    @property
    def n_nodes(self) -> int:
        return self.nodes.shape[0]


_KUHN = np.array([[0, 1, 3, 7], [0, 1, 5, 7], [0, 2, 3, 7], [0, 2, 6, 7], [0, 4, 5, 7], [0, 4, 6, 7]])


def _grid_mesh(inside, lo, hi, h) -> Mesh:
    n = np.maximum(np.ceil((np.asarray(hi) - np.asarray(lo)) / h).astype(int), 1)
    ax = [np.linspace(lo[d], lo[d] + n[d] * h, n[d] + 1) for d in range(3)]
    nx, ny, nz = (len(a) for a in ax)
    I, J, K = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()

    def vid(di, dj, dk):
        return ((I + di) * ny + (J + dj)) * nz + (K + dk)

    corners = np.stack([vid((c >> 2) & 1, (c >> 1) & 1, c & 1) for c in range(8)], axis=1)
    tets = corners[:, _KUHN].reshape(-1, 4)
    P = np.stack(np.meshgrid(*ax, indexing="ij"), axis=-1).reshape(-1, 3)
    cent = P[tets].mean(axis=1)
    keep = inside(cent)
    tets = tets[keep]
    used = np.unique(tets.ravel())
    remap = -np.ones(P.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.size)
    return Mesh(P[used].copy(), remap[tets].astype(np.int32))


def _fit_mesh(inside, lo, hi, volume, target_nodes) -> Mesh:
    h = (volume / max(target_nodes, 8)) ** (1.0 / 3.0)
    mesh = _grid_mesh(inside, lo, hi, h)
    for _ in range(3):
        ratio = mesh.n_nodes / target_nodes
        if abs(ratio - 1) < 0.03:
            break
        h *= ratio ** (1.0 / 3.0)
        mesh = _grid_mesh(inside, lo, hi, h)
    return mesh


def cylinder(n_nodes=20_000, radius=0.04, height=0.08) -> Mesh:
    def inside(c):
        return (c[:, 0] ** 2 + c[:, 1] ** 2 <= radius ** 2) & (np.abs(c[:, 2]) <= height / 2)
    return _fit_mesh(inside, (-radius, -radius, -height / 2), (radius, radius, height / 2),
                     np.pi * radius ** 2 * height, n_nodes)


def tube(n_nodes=200_000, radius=0.012, length=0.1) -> Mesh:
    return cylinder(n_nodes, radius, length)


def ellipsoid(n_nodes=500_000, axes=(0.06, 0.05, 0.04)) -> Mesh:
    a = np.asarray(axes)

    def inside(c):
        return ((c / a) ** 2).sum(axis=1) <= 1.0
    return _fit_mesh(inside, -a, a, 4.0 / 3.0 * np.pi * np.prod(a), n_nodes)


def tissue(n, seed=0):
    """T1 ~ U[800, 1200] ms, T2 ~ U[50, 100] ms (float32)."""
    rng = np.random.default_rng(seed)
    T1 = rng.uniform(800.0, 1200.0, n).astype(np.float32)
    T2 = rng.uniform(50.0, 100.0, n).astype(np.float32)
    return T1, T2


# --------------------------------------------------------------- sequences --

@dataclass
class Block:
    """One discretised sequence block: the arrays BlochSolver passes to
    solve_mri (Bloch.py:339-352).  `dt` has dt[0] = absolute start time."""
    times: np.ndarray   # (n_t,) float64, ms
    rf: np.ndarray      # (n_t,) complex64, mT
    G: np.ndarray       # (n_t, 3) float32, mT/m
    empty: bool = False
    store_magnetization: bool = False

    @property
    def dt(self) -> np.ndarray:
        return np.diff(self.times, prepend=0.0)

    @property
    def t0(self) -> float:
        return float(self.times[0])


def hard_pulse_block(t0, flip_deg, tr, rf_dur=0.1, dt_rf=0.01, dt=0.1, grad=None, store=False) -> Block:
    """RF hard pulse of `flip_deg` at t0, then free precession until t0 + tr.
    `grad`: optional (G_xyz, start, duration) spoiler/encoding lobe in mT/m."""
    n_rf = int(round(rf_dur / dt_rf))
    t_rf = t0 + dt_rf * np.arange(n_rf + 1)
    t_free = t0 + rf_dur + dt * np.arange(1, int(round((tr - rf_dur) / dt)) + 1)
    times = np.concatenate([t_rf, t_free])
    amp = np.deg2rad(flip_deg) / (GAMMA * rf_dur)  # mT, constant over the pulse
    rf = np.zeros(times.size, np.complex64)
    rf[1:n_rf + 1] = amp
    G = np.zeros((times.size, 3), np.float32)
    if grad is not None:
        g, gs, gd = grad
        on = (times > t0 + gs) & (times <= t0 + gs + gd)
        G[on] = np.asarray(g, np.float32)
    return Block(times, rf, G, store_magnetization=store)


def spamm_block(t0, tag_spacing=0.008, axis=0, rf_dur=0.1, dt_rf=0.01, lobe=0.5, dt=0.01, tail=1.0) -> Block:
    """SPAMM tagging as examples/spamm.py:116-125 builds it: a 90-degree hard
    pulse, a gradient lobe along `axis` of area ke / gamma with
    ke = 2 pi / tag_spacing (785.4 rad/m at 8 mm), a second 90-degree hard
    pulse (same phase), then free precession for `tail` ms; Mz is left
    modulated as -cos(ke x)."""
    n_rf = int(round(rf_dur / dt_rf))
    ke = 2.0 * np.pi / tag_spacing
    g = ke / (GAMMA * lobe)  # mT/m
    t_rf1 = t0 + dt_rf * np.arange(n_rf + 1)
    t_lobe = t_rf1[-1] + dt * np.arange(1, int(round(lobe / dt)) + 1)
    t_rf2 = t_lobe[-1] + dt_rf * np.arange(1, n_rf + 1)
    t_tail = t_rf2[-1] + 0.1 * np.arange(1, int(round(tail / 0.1)) + 1)
    times = np.concatenate([t_rf1, t_lobe, t_rf2, t_tail])
    amp = np.deg2rad(90.0) / (GAMMA * rf_dur)
    rf = np.zeros(times.size, np.complex64)
    rf[1:n_rf + 1] = amp
    i2 = n_rf + 1 + t_lobe.size
    rf[i2:i2 + n_rf] = amp
    G = np.zeros((times.size, 3), np.float32)
    G[n_rf + 1:n_rf + 1 + t_lobe.size, axis] = g
    return Block(times, rf, G)


def spoiled_gre(n_pulses=20, flip_deg=15.0, tr=5.0) -> list[Block]:
    return [hard_pulse_block(i * tr, flip_deg, tr, store=(i == n_pulses - 1)) for i in range(n_pulses)]


def pc_imaging_block(t0, enc_dir, venc=1.5, flip_deg=15.0, tr=5.0, lobe=0.5, dt=0.01) -> Block:
    """Phase-contrast block: hard pulse, then a bipolar lobe pair along
    enc_dir (zero for the reference encoding) sized so that a velocity of
    `venc` m/s accrues a phase of pi: gamma G lobe^2 * (venc / 1000) = pi."""
    n_rf = 10
    rf_dur = 0.1
    enc = np.asarray(enc_dir, np.float64)
    g = 0.0 if not np.any(enc) else np.pi / (GAMMA * lobe ** 2 * (venc / 1000.0))
    t_rf = t0 + (rf_dur / n_rf) * np.arange(n_rf + 1)
    t_enc = t0 + rf_dur + dt * np.arange(1, int(round(2 * lobe / dt)) + 1)
    t_rest = t_enc[-1] + 0.1 * np.arange(1, int(round((tr - rf_dur - 2 * lobe) / 0.1)) + 1)
    times = np.concatenate([t_rf, t_enc, t_rest])
    rf = np.zeros(times.size, np.complex64)
    rf[1:n_rf + 1] = np.deg2rad(flip_deg) / (GAMMA * rf_dur)
    G = np.zeros((times.size, 3), np.float32)
    first = (times > t0 + rf_dur) & (times <= t0 + rf_dur + lobe)
    second = (times > t0 + rf_dur + lobe) & (times <= t0 + rf_dur + 2 * lobe)
    G[first] = (g * enc).astype(np.float32)
    G[second] = (-g * enc).astype(np.float32)
    return Block(times, rf, G, store_magnetization=True)


PC_ENCODINGS = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]


# ------------------------------------------------------------ trajectories --

@dataclass
class Trajectory:
    kx: np.ndarray   # (n_ro, n_lines, n_kz) float32, 1/m
    ky: np.ndarray
    kz: np.ndarray
    t: np.ndarray    # (n_ro, n_lines, n_kz) float32, ms

    @property
    def points(self):
        return (self.kx, self.ky, self.kz)

    @property
    def shape(self):
        return self.kx.shape

    @property
    def n_samples(self) -> int:
        return int(np.prod(self.kx.shape))


def cartesian(res=(96, 96, 32), fov=(0.1, 0.1, 0.1), t_start=2.0, dwell=1.0 / 128.0) -> Trajectory:
    """Cartesian stack: kx along the readout, ky per line, kz per slice; the
    sample time depends on the readout index only (KSpaceTraj.py:180-220)."""
    n_ro, n_ph, n_kz = res
    dk = 1.0 / np.asarray(fov, np.float64)
    kx = (np.arange(n_ro) - n_ro // 2) * dk[0]
    ky = (np.arange(n_ph) - n_ph // 2) * dk[1]
    kz = (np.arange(n_kz) - n_kz // 2) * dk[2]
    KX, KY, KZ = np.meshgrid(kx, ky, kz, indexing="ij")
    t = t_start + dwell * np.arange(n_ro)
    T = np.broadcast_to(t[:, None, None], KX.shape)
    f = np.float32
    return Trajectory(KX.astype(f), KY.astype(f), KZ.astype(f), np.ascontiguousarray(T, dtype=f))


def radial3d(n_ro=256, n_spokes=4096, kmax=500.0, t_start=2.0, dwell=1.0 / 128.0) -> Trajectory:
    """Centre-out 3-D radial spokes along Fibonacci-sphere directions; all
    spokes share the readout clock, so times depend on the readout index."""
    i = np.arange(n_spokes) + 0.5
    phi = np.arccos(1 - 2 * i / n_spokes)
    theta = np.pi * (1 + 5 ** 0.5) * i
    d = np.stack([np.cos(theta) * np.sin(phi), np.sin(theta) * np.sin(phi), np.cos(phi)], axis=1)
    r = kmax * np.arange(n_ro) / max(n_ro - 1, 1)
    K = r[:, None, None] * d[None, :, :]
    t = t_start + dwell * np.arange(n_ro)
    T = np.broadcast_to(t[:, None], (n_ro, n_spokes))[..., None]
    f = np.float32
    return Trajectory(K[..., 0:1].astype(f), K[..., 1:2].astype(f), K[..., 2:3].astype(f),
                      np.ascontiguousarray(T, dtype=f))


def spiral_stack(n_ro=2048, n_interleaves=8, n_kz=8, fov=0.1, kmax=300.0, t_start=2.0,
                 dwell=1.0 / 128.0) -> Trajectory:
    """Archimedean spiral interleaves stacked along kz."""
    s = np.arange(n_ro) / max(n_ro - 1, 1)
    turns = kmax * fov / n_interleaves
    ang = 2 * np.pi * turns * s
    kr = kmax * s
    base = np.stack([kr * np.cos(ang), kr * np.sin(ang)], axis=1)
    KX = np.zeros((n_ro, n_interleaves, n_kz))
    KY = np.zeros_like(KX)
    KZ = np.zeros_like(KX)
    kz = (np.arange(n_kz) - n_kz // 2) / fov
    for j in range(n_interleaves):
        a = 2 * np.pi * j / n_interleaves
        c, sn = np.cos(a), np.sin(a)
        KX[:, j, :] = (c * base[:, 0] - sn * base[:, 1])[:, None]
        KY[:, j, :] = (sn * base[:, 0] + c * base[:, 1])[:, None]
        KZ[:, j, :] = kz[None, :]
    t = t_start + dwell * np.arange(n_ro)
    T = np.broadcast_to(t[:, None, None], KX.shape)
    f = np.float32
    return Trajectory(KX.astype(f), KY.astype(f), KZ.astype(f), np.ascontiguousarray(T, dtype=f))


# ------------------------------------------------------------------ motion --

def poiseuille_velocity(nodes, radius, v_max=1.0, period=1000.0, n_frames=20):
    """Rank-1 velocity-mode motion of v = v_max (1 - rho^2/R^2) z in m/ms:
    the displacement at time t is v t, the form of a PODVelocity
    (Motion.py:272-290)."""
    from .motion import SplineMotion
    rho2 = nodes[:, 0] ** 2 + nodes[:, 1] ** 2
    v = np.zeros((nodes.shape[0], 3, 1))
    v[:, 2, 0] = v_max * np.clip(1 - rho2 / radius ** 2, 0, None) / 1000.0
    times = np.linspace(0.0, period, n_frames).astype(np.float32)
    w = np.ones((n_frames, 1))
    return SplineMotion.from_samples(v, times, w, periodic=True, velocity=True)


def sinusoidal_pod(n_nodes, n_modes=10, amp=1e-3, period=800.0, n_frames=40, seed=2):
    """Mode motion with Phi ~ N(0, amp) metres and a_m(t) = sin(2 pi t / period + psi_m),
    periodic in `period`."""
    from .motion import SplineMotion
    rng = np.random.default_rng(seed)
    modes = rng.normal(0.0, amp, (n_nodes, 3, n_modes))
    psi = rng.uniform(0, 2 * np.pi, n_modes)
    times = np.linspace(0.0, period, n_frames)
    w = np.sin(2 * np.pi * times[:, None] / period + psi[None, :])
    return SplineMotion.from_samples(modes, times, w, periodic=True)


def coil_maps(nodes, n_coils=8, sigma=0.08, ring=0.15, seed=3) -> np.ndarray:
    """Smooth Gaussian coil sensitivities (N, n_coils) complex64."""
    rng = np.random.default_rng(seed)
    ang = 2 * np.pi * np.arange(n_coils) / n_coils
    centres = np.stack([ring * np.cos(ang), ring * np.sin(ang), np.zeros(n_coils)], axis=1)
    psi = rng.uniform(0, 2 * np.pi, n_coils)
    d2 = ((nodes[:, None, :] - centres[None, :, :]) ** 2).sum(-1)
    return (np.exp(-d2 / (2 * sigma ** 2)) * np.exp(1j * psi)[None, :]).astype(np.complex64)


def off_resonance(n, sigma_hz=20.0, seed=1) -> np.ndarray:
    """phi ~ N(0, sigma) Hz as rad/ms (float32)."""
    rng = np.random.default_rng(seed)
    return (2 * np.pi * rng.normal(0.0, sigma_hz, n) / 1000.0).astype(np.float32)


@dataclass
class SignalCase:
    """Inputs of one Signal call as numpy arrays (float32 unless stated)."""
    mesh: Mesh
    M: object                      # scipy sparse (N, N)
    traj: Trajectory
    r0: np.ndarray
    phi: np.ndarray
    T2: np.ndarray
    Mxy: np.ndarray                # (N, V) complex64
    pod: object = None
    meta: dict = field(default_factory=dict)
