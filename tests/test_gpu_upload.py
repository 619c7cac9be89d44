"""Host-to-device staging of the shims' inputs (ops.upload_many): one pinned
buffer and one copy per call must give the same tensors as a per-array
`torch.from_numpy(a).to(device, dtype)`, for mixed dtypes, empty and
non-contiguous arrays, arrays large enough for the threaded copy, and
back-to-back calls that reuse the staging buffer."""
import numpy as np
import pytest
import torch

from feelmri_b200 import ops

pytestmark = pytest.mark.gpu


def _items(rng, big):
    n = 300_000 if big else 37
    return [
        (rng.integers(-5, 5, n + 1).astype(np.int64), torch.int32),
        (rng.normal(size=(n, 3)), torch.float32),
        (rng.normal(size=2 * n)[::2], torch.float32),  # non-contiguous view
        (np.zeros(0, np.float32), torch.float32),
        ((rng.normal(size=(n, 4)) + 1j * rng.normal(size=(n, 4))).astype(np.complex64), torch.complex64),
        (rng.normal(size=n).astype(np.float32), torch.float64),
    ]


@pytest.mark.parametrize("big", [False, True])
def test_upload_many_matches_per_array_copies(cuda, big):
    rng = np.random.default_rng(7)
    for _ in range(3):  # the staging buffer is reused by the later calls
        items = _items(rng, big)
        got = ops.upload_many(items, cuda)
        torch.cuda.synchronize(cuda)
        for (a, dt), t in zip(items, got):
            want = torch.from_numpy(np.ascontiguousarray(a)).to(device=cuda, dtype=dt)
            assert t.dtype == dt and t.device == want.device and tuple(t.shape) == tuple(want.shape)
            assert torch.equal(t, want)


def test_upload_many_results_are_independent(cuda):
    """Tensors of one call are separate allocations from the next call's."""
    a = ops.upload_many([(np.arange(10, dtype=np.float32), torch.float32)], cuda)[0]
    b = ops.upload_many([(np.full(10, 3.0, np.float32), torch.float32)], cuda)[0]
    torch.cuda.synchronize(cuda)
    assert torch.equal(a.cpu(), torch.arange(10, dtype=torch.float32))
    assert torch.equal(b.cpu(), torch.full((10,), 3.0))
