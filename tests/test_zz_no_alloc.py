"""The non-allocating shell sums, called through the C ABI, against the allocating
entry point `djb_power_spectrum` on the same field, twice in a row (the second call
reuses the shared scratch left by the first). Collected last on purpose.

Callers that cannot allocate (under an external memory pool, or in a step loop that
must not synchronise through the allocator) use this entry point; it must agree with
the ordinary one."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

PK_TOL = 1e-4  # per-bin tolerance of the P(k) parity tests


@pytest.fixture(scope="module")
def djb(cuda_device):
    import djb200
    return djb200


def _field(res, seed):
    rng = np.random.default_rng(seed)
    f = rng.standard_normal((res, res, res)).astype(np.float32)
    f[2:9, 5:11, 3:7] += 3.0
    return f


@pytest.mark.parametrize("res,bins,log", [(48, 32, True), (64, 20, False)])
def test_noalloc_matches_allocating_entry_point(djb, res, bins, log):
    import torch

    from djb200 import power
    L = 250.0
    f = _field(res, 17 + res)                      # logical [ix, iy, iz]
    k0, p0, n0 = djb.evaluate_power_spectrum(f, L, bins=bins, logarithmic=log)
    # the same field in device memory, stored [iz, iy, ix] (x fastest), transformed there
    spec = torch.fft.rfftn(torch.from_numpy(np.ascontiguousarray(f.transpose(2, 1, 0))).cuda(),
                           dim=(0, 1, 2)).contiguous()
    torch.cuda.synchronize()
    for _ in range(2):
        before = torch.cuda.current_device()
        k, p, nm = power.power_spectrum_shells_noalloc(spec, L, bins=bins, logarithmic=log)
        assert torch.cuda.current_device() == before   # the caller's device is left as it was
        assert np.array_equal(nm, n0)
        assert rel(k, k0) < 1e-13
        nz = n0 > 0
        assert np.max(np.abs(p[nz] / p0[nz] - 1)) < PK_TOL
        assert np.all(p[~nz] == 0)


def test_noalloc_rejects_too_many_bins(djb):
    import torch

    from djb200 import power
    spec = torch.zeros((16, 16, 9), dtype=torch.complex64, device="cuda")
    with pytest.raises(djb.DJBInvalidOption, match="exceeds the 512 bins"):
        power.power_spectrum_shells_noalloc(spec, 100.0, bins=513)


def test_noalloc_rejects_wrong_dtype_or_host_tensor(djb):
    """Only complex64 device spectra are read; anything else raises before the C call."""
    import torch

    from djb200 import power
    with pytest.raises(ValueError, match="complex64 CUDA tensor"):
        power.power_spectrum_shells_noalloc(torch.zeros((16, 16, 9), dtype=torch.complex128, device="cuda"), 100.0)
    with pytest.raises(ValueError, match="complex64 CUDA tensor"):
        power.power_spectrum_shells_noalloc(torch.zeros((16, 16, 9), dtype=torch.complex64), 100.0)
