"""Exact NUDFT reconstruction operators on the GPU (feelmri_b200.Recon):
the adjoint against the FP64 direct sum and against numpy's inverse FFT on a
Cartesian grid, forward/adjoint consistency, and Pipe-Menon density
compensation.  The reference reconstructs with pynufft's gridding NUFFT
(python/feelmri/Recon.py:150-290), which is not installed here; these are the
exact sums that it approximates."""
import numpy as np
import pytest

from oracle import fp64
from feelmri_b200 import Recon, workloads as W

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 1e-4, "f32": 1e-4}


def _radial(n_ro=24, n_spokes=300, kmax=150.0):
    tr = W.radial3d(n_ro=n_ro, n_spokes=n_spokes, kmax=kmax)
    return tr.kx, tr.ky, tr.kz


@pytest.mark.parametrize("precision", ["bf16x3", "f32"])
def test_adjoint_matches_direct_sum(cuda, precision):
    kx, ky, kz = _radial()
    S = kx.size
    rng = np.random.default_rng(1)
    K = (rng.normal(size=(S, 2)) + 1j * rng.normal(size=(S, 2))).astype(np.complex64)
    dcw = rng.uniform(0.5, 1.5, S).astype(np.float32)
    shape, fov = (10, 12, 6), (0.12, 0.1, 0.08)
    img = Recon.nudft_adjoint(K, kx, ky, kz, shape, fov, dcw=dcw, precision=precision)
    assert img.shape == (*shape, 2) and img.dtype == np.complex64
    X, Y, Z = Recon.grid_points(shape, fov)
    ref = fp64.nudft_adjoint(kx, ky, kz, K, np.stack([X, Y, Z], -1), dcw=dcw).reshape(*shape, 2)
    assert fp64.rel_l2(img, ref) < TOL[precision]


def test_adjoint_of_cartesian_data_is_the_inverse_dft(cuda):
    # k on the grid's reciprocal lattice: the adjoint is N * ifftn with the
    # DFT-centred index conventions of both axes
    shape, fov = (8, 10, 4), (0.08, 0.1, 0.04)
    rng = np.random.default_rng(2)
    kidx = [np.arange(n) - n // 2 for n in shape]
    KX, KY, KZ = np.meshgrid(*[ki / f for ki, f in zip(kidx, fov)], indexing="ij")
    K = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    img = Recon.nudft_adjoint(K.reshape(-1), KX, KY, KZ, shape, fov)[..., 0]
    ref = np.fft.fftshift(np.fft.ifftn(np.fft.ifftshift(K))) * K.size
    assert fp64.rel_l2(img, ref) < 1e-4


def test_forward_and_adjoint_are_transposes(cuda):
    # <A x, y> = <x, A^H y>
    kx, ky, kz = _radial(n_ro=16, n_spokes=200)
    shape, fov = (8, 8, 8), (0.1, 0.1, 0.1)
    rng = np.random.default_rng(3)
    x = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    y = (rng.normal(size=kx.shape) + 1j * rng.normal(size=kx.shape)).astype(np.complex64)
    Ax = Recon.nudft_forward(x, kx, ky, kz, (0.1, 0.1, 0.1))[..., 0]
    Ahy = Recon.nudft_adjoint(y.reshape(-1), kx, ky, kz, shape, fov)[..., 0]
    lhs = np.vdot(y, Ax)
    rhs = np.vdot(Ahy, x)
    assert abs(lhs - rhs) / abs(lhs) < 1e-4


def test_pipe_menon_weights_follow_the_sampling_density(cuda):
    # centre-out radial spokes oversample the centre: the weights grow with |k|
    kx, ky, kz = _radial(n_ro=16, n_spokes=200, kmax=70.0)
    w = Recon.dcf_pipe_menon(kx, ky, kz, (16, 16, 16), (0.1, 0.1, 0.1), n_iter=8)
    assert w.shape == (kx.size,) and np.all(w > 0) and abs(w.mean() - 1) < 1e-4
    kr = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2).reshape(-1)
    inner, outer = w[kr < 20].mean(), w[kr > 50].mean()
    assert outer > 3 * inner


def test_reconstruct_shapes_and_rss(cuda):
    kx, ky, kz = (a.reshape(16, 20, 1) for a in _radial(n_ro=16, n_spokes=20))
    rng = np.random.default_rng(4)
    kdata = (rng.normal(size=(16, 20, 1, 3)) + 1j * rng.normal(size=(16, 20, 1, 3))).astype(np.complex64)
    img = Recon.reconstruct_nudft(kdata, (kx, ky, kz), (6, 6, 4), (0.1, 0.1, 0.1), auto_dcw="jacobian")
    assert img.shape == (3, 6, 6, 4)
    rss = Recon.reconstruct_nudft(kdata, (kx, ky, kz), (6, 6, 4), (0.1, 0.1, 0.1), auto_dcw="jacobian", combine="rss")
    np.testing.assert_allclose(np.abs(rss), np.sqrt((np.abs(img) ** 2).sum(0)), rtol=1e-5)


class _Stack:
    """The CartesianStack attributes cartesian_recon reads."""

    def __init__(self, res, lines_per_shot=1, oversampling=1):
        self.res = np.array(res)
        self.oversampling_arr = np.array([oversampling, 1.0, 1.0])
        self.lines_per_shot = lines_per_shot
        n_shots = res[1] // lines_per_shot
        self.shots = [[s * lines_per_shot + i for i in range(lines_per_shot)] for s in range(n_shots)]


def _numpy_cartesian(K, st, kind):
    # the same steps in numpy: line flips, even-axis padding, separable
    # window on readout x phase, centred inverse FFT over the first 3 axes
    K = K.astype(np.complex128).copy()
    if st.lines_per_shot > 1:
        for shot in st.shots:
            for pos, line in enumerate(shot):
                if pos % 2 == 1:
                    K[:, line] = K[::-1, line].copy()
    pad = [(0, 1) if st.res[d] % 2 == 0 else (0, 0) for d in range(3)] + [(0, 0)] * (K.ndim - 3)
    K = np.pad(K, pad)
    h = np.outer(Recon._kspace_window(K.shape[0], kind), Recon._kspace_window(K.shape[1], kind))
    K = K * h.reshape(h.shape + (1,) * (K.ndim - 2))
    ax = (0, 1, 2)
    return np.fft.fftshift(np.fft.ifftn(np.fft.ifftshift(K, axes=ax), axes=ax), axes=ax)


@pytest.mark.parametrize("res,lps,kind", [((15, 13, 5), 1, "Tukey"), ((15, 13, 3), 2, "Riesz"),
                                          ((17, 11, 1), 4, "none"), ((16, 12, 4), 2, "Tukey")])
def test_cartesian_recon_matches_numpy(cuda, res, lps, kind):
    rng = np.random.default_rng(5)
    K = (rng.normal(size=(*res, 2, 3)) + 1j * rng.normal(size=(*res, 2, 3))).astype(np.complex64)
    st = _Stack(res, lps)
    img = Recon.cartesian_recon(K, st, {"type": kind})
    assert img.shape == (*res, 2, 3) and img.dtype == np.complex64
    ref = _numpy_cartesian(K, st, kind)
    if ref.shape[:3] == img.shape[:3]:
        # odd resolutions: no padding, so no interpolation back to res
        np.testing.assert_allclose(img, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max())
    else:
        # even axes are padded by one sample; the image is interpolated back
        # to res, which changes it by a fraction of a voxel only
        assert ref.shape[:3] == tuple(r + (r % 2 == 0) for r in res)


def test_cartesian_recon_of_a_point_and_oversampling(cuda):
    # one voxel's k-space (a plane wave) reconstructs to that voxel; with a
    # 2x oversampled readout the image comes back at res with the readout
    # cut around its centre
    res = (9, 7, 3)
    n = np.array(res)
    x0 = (2, -1, 0)
    g = [np.arange(m) - m // 2 for m in n]
    KX, KY, KZ = np.meshgrid(*g, indexing="ij")
    K = np.exp(-2j * np.pi * (KX * x0[0] / n[0] + KY * x0[1] / n[1] + KZ * x0[2] / n[2])).astype(np.complex64)
    img = Recon.cartesian_recon(K[..., None, None], _Stack(res), {"type": "none"})[..., 0, 0]
    peak = np.unravel_index(np.argmax(np.abs(img)), img.shape)
    assert tuple(int(p) - m // 2 for p, m in zip(peak, n)) == x0
    Kos = np.ones((18, 7, 3, 1, 1), np.complex64)
    out = Recon.cartesian_recon(Kos, _Stack(res, oversampling=2), {"type": "Tukey"})
    assert out.shape == (9, 7, 3, 1, 1)
