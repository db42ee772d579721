"""The library's radix sort (per-frame prefix-endpoint structure) against a
stable sort of the keys' high 32 bits in numpy, across tile boundaries and
with the key forms the renderer makes: Morton code << 32 | index, all ones
for an absent entry, many equal codes."""
import ctypes

import numpy as np
import pytest
import torch

from crisoptix_b200 import _abi

pytestmark = pytest.mark.gpu


def gpu_sort(keys: np.ndarray) -> np.ndarray:
    lib = _abi.load()
    n = len(keys)
    d_in = torch.from_numpy(keys.view(np.int64)).cuda()
    d_out = torch.full((max(n, 1),), -1, dtype=torch.int64, device="cuda")
    tb = lib.crisb_selftest_sort_temp_bytes(n)
    tmp = torch.empty(tb, dtype=torch.uint8, device="cuda")
    _abi.check(lib.crisb_selftest_sort(ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()), n,
                                       ctypes.c_void_p(tmp.data_ptr()), tb, None))
    torch.cuda.synchronize()
    assert (d_in.cpu().numpy().view(np.uint64) == keys).all()  # input untouched
    return d_out.cpu().numpy().view(np.uint64)[:n]


@pytest.mark.parametrize("n", [1, 2, 255, 2047, 2048, 2049, 6143, 100003, 2073600])
def test_sort_matches_stable_numpy_sort(cuda_device, n):
    rng = np.random.default_rng(n)
    morton = rng.integers(0, 1 << 30, n, dtype=np.uint64)
    tie = rng.random(n) < 0.3
    morton[tie] = rng.integers(0, 64, int(tie.sum()), dtype=np.uint64)  # many equal codes
    keys = (morton << np.uint64(32)) | np.arange(n, dtype=np.uint64)
    keys[rng.random(n) < 0.1] = np.uint64(0xFFFFFFFFFFFFFFFF)  # absent entries
    want = keys[np.argsort(keys >> np.uint64(32), kind="stable")]
    got = gpu_sort(keys)
    assert (got == want).all()
    assert (np.sort(keys) == got).all()  # the same as sorting all 64 bits
