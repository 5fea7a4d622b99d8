"""argot_b200_scan_blocks_static: the ray-offset scan for callers that
cannot allocate device memory (its scratch is a fixed device array).  Its
output must equal the allocating argot_b200_scan_blocks exactly (integer
prefix sums), on consecutive calls that share the array.  This file is named
to be collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_BLOCKS = 16_777_216


def _scan(lib, fn, counts, base):
    import torch
    nb = counts.numel()
    off = torch.full((nb + 1,), -1, dtype=torch.int64, device="cuda")
    tot = C.c_uint64()
    rc = getattr(lib, fn)(counts.data_ptr(), nb, base, off.data_ptr(), C.byref(tot),
                          torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rc, off.cpu().numpy(), tot.value


def test_static_scan_equals_allocating_scan(cuda_ok):
    import torch
    from argot_b200 import _lib as L
    lib = L.load()
    rng = np.random.default_rng(12)
    for nb, base in ((1, 0), (2048 * 3 + 5, 7), (300_001, 123_456_789), (2_000_003, 0)):
        for call in range(2):  # two calls in a row share the device array
            counts = torch.from_numpy(rng.integers(0, 1000, nb).astype(np.int64)).cuda()
            rc0, want, tot0 = _scan(lib, "argot_b200_scan_blocks", counts, base)
            rc1, got, tot1 = _scan(lib, "argot_b200_scan_blocks_static", counts, base)
            assert rc0 == 0 and rc1 == 0
            assert np.array_equal(got, want), (nb, call)
            assert tot1 == tot0 == base + int(counts.sum().item())


def test_static_scan_largest_size(cuda_ok):
    """nb at the limit: the whole scratch array (8192 tiles) in use."""
    import torch
    from argot_b200 import _lib as L
    lib = L.load()
    counts = torch.randint(0, 300, (MAX_BLOCKS,), dtype=torch.int64, device="cuda")
    rc0, want, tot0 = _scan(lib, "argot_b200_scan_blocks", counts, 11)
    rc1, got, tot1 = _scan(lib, "argot_b200_scan_blocks_static", counts, 11)
    assert rc0 == 0 and rc1 == 0
    assert np.array_equal(got, want)
    assert tot1 == tot0 == 11 + int(counts.sum().item())


def test_static_scan_rejects_oversize(cuda_ok):
    """One block past the limit: rejected before any launch.  The buffers
    are sized for the request, so even a launch would stay in bounds."""
    import torch
    from argot_b200 import _lib as L
    lib = L.load()
    nb = MAX_BLOCKS + 1
    counts = torch.ones(nb, dtype=torch.int64, device="cuda")
    off = torch.zeros(nb + 1, dtype=torch.int64, device="cuda")
    tot = C.c_uint64(99)
    rc = lib.argot_b200_scan_blocks_static(counts.data_ptr(), nb, 0, off.data_ptr(),
                                           C.byref(tot), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == L.EINVAL
    assert tot.value == 99  # nothing ran
    assert int(off.abs().sum().item()) == 0
