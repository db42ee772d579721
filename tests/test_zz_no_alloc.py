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
