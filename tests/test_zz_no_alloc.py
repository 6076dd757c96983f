"""The allocation-free threshold entry point.

Callers that may not allocate device memory (a host that owns the GPU's
memory through its own pool, a real-time loop that cannot absorb
cudaMalloc's synchronisation) call wema_cuda_threshold_flat_noalloc, whose
scratch is a fixed array inside the library.  Its result must equal the
allocating entry point's bit for bit - the threshold decides amplification
masks, so any difference is a parity failure - on consecutive calls (the
shared scratch keeps the previous call's contents).  This file sorts last so
a run that stops at the first failure has run everything else first.
"""
import numpy as np
import pytest

from wema_b200 import cuda as wc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("needs a CUDA device")
    return torch


def _bits(x):
    return np.asarray([x], np.float32).view(np.uint32)[0]


@pytest.mark.parametrize("n", [1, 7, 1000, 4131360, 1 << 24])
def test_noalloc_matches_allocating_entry_point(torch_cuda, n):
    torch = torch_cuda
    rng = np.random.default_rng(n)
    arrays = [
        (rng.standard_normal(n) * 10.0 ** rng.integers(-6, 3, n)).astype(np.float32),
        np.full(n, 0.1, np.float32),
    ]
    for x in arrays:            # two calls in a row share the static scratch
        d = torch.from_numpy(x).cuda()
        for form in (wc.THR_SINGLE, wc.THR_BATCH):
            t0, s0 = wc.threshold_flat(d, form)
            t1, s1 = wc.threshold_flat_noalloc(d, form)
            assert _bits(t1) == _bits(t0) and _bits(s1) == _bits(s0)


def test_noalloc_rejects_oversize(torch_cuda):
    torch = torch_cuda
    d = torch.zeros(16, device="cuda")
    rc = wc.lib().wema_cuda_threshold_flat_noalloc(d.data_ptr(), (1 << 24) + 1, 0,
                                                   d.data_ptr(), None, None)
    assert rc == -1
    assert "exceeds" in wc.last_error()
