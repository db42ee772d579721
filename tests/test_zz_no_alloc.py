"""crisb_endpoint_search_noalloc, the allocation-free endpoint search, must
return exactly what crisb_endpoint_search returns.

It exists for callers that may not allocate device memory while they run
(engines that reserve all device memory up front, plugin hosts without an
allocator).  Its scratch is a static device array shared by all calls, so
the test makes two calls in a row with different inputs: the second must not
see anything left over from the first.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

from crisoptix_b200 import _abi
from test_endpoint_search_gpu import gpu_search, make_case

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_search_twice(cuda_device):
    cases = [(make_case(101, n_entries=20000, n_queries=4000), 8),
             (make_case(202, n_entries=5000, n_queries=3000), 31)]
    for (entries, queries), k in cases:
        ref, rc = gpu_search(entries, queries, k, "crisb_endpoint_search")
        got, gc = gpu_search(entries, queries, k, "crisb_endpoint_search_noalloc")
        assert (gc == rc).all()
        assert got.tobytes() == ref.tobytes()
        assert rc.max() > 0


def _pool_used_bytes() -> int:
    """Bytes in use in the current device's default stream-ordered pool."""
    from cuda.bindings import runtime as cr

    err, dev = cr.cudaGetDevice()
    assert err == cr.cudaError_t.cudaSuccess
    err, pool = cr.cudaDeviceGetDefaultMemPool(dev)
    assert err == cr.cudaError_t.cudaSuccess
    err, used = cr.cudaMemPoolGetAttribute(pool, cr.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    assert err == cr.cudaError_t.cudaSuccess
    return int(used)


def test_noalloc_call_allocates_nothing(cuda_device):
    """Around one synchronised call, neither the stream-ordered pool's bytes
    in use nor the device's free memory may change (everything the call
    touches is allocated before the first reading)."""
    lib = _abi.load()
    entries, queries = make_case(303, n_entries=8000, n_queries=2000)
    k = 8
    e = torch.from_numpy(entries).cuda()
    q = torch.from_numpy(queries).cuda()
    out = torch.zeros((len(queries), k, 2), dtype=torch.int32, device="cuda")
    cnt = torch.zeros(len(queries), dtype=torch.int32, device="cuda")
    args = (ctypes.c_void_p(e.data_ptr()), len(entries), ctypes.c_void_p(q.data_ptr()), len(queries), k,
            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()), None)
    _abi.check(lib.crisb_endpoint_search_noalloc(*args))  # first call: address lookup, module load
    torch.cuda.synchronize()
    used0, free0 = _pool_used_bytes(), torch.cuda.mem_get_info()[0]
    _abi.check(lib.crisb_endpoint_search_noalloc(*args))
    torch.cuda.synchronize()
    assert _pool_used_bytes() == used0
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_oversized_input(cuda_device):
    lib = _abi.load()
    n = 32768 + 1
    e = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    q = torch.zeros((1, 3), dtype=torch.float32, device="cuda")
    out = torch.zeros((1, 4, 2), dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.crisb_endpoint_search_noalloc(ctypes.c_void_p(e.data_ptr()), n, ctypes.c_void_p(q.data_ptr()), 1, 4,
                                           ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()), None)
    assert rc == _abi.ERR_INVALID_ARGUMENT
    buf = ctypes.create_string_buffer(256)
    lib.crisb_last_error(buf, 256)
    assert b"exceeds the maximum" in buf.value
