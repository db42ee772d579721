"""The standalone prefix-endpoint search (crisb_endpoint_search) against a
float32 brute force over every entry (same distance arithmetic, so the lists
must match exactly)."""
import ctypes

import numpy as np
import pytest
import torch

from crisoptix_b200 import _abi

pytestmark = pytest.mark.gpu


def brute_force(entries: np.ndarray, queries: np.ndarray, k: int):
    e = entries.astype(np.float32)
    valid = (e[:, 3] >= 0) & np.isfinite(e[:, :3]).all(axis=1)
    out = np.zeros((len(queries), k), _abi.NEIGHBOR_DTYPE)
    cnt = np.zeros(len(queries), np.uint32)
    for qi, q in enumerate(queries.astype(np.float32)):
        dx = e[:, 0] - q[0]
        dy = e[:, 1] - q[1]
        dz = e[:, 2] - q[2]
        d = np.sqrt((dx * dx + dy * dy) + dz * dz).astype(np.float32)
        ok = np.nonzero(valid & ~(d > e[:, 3]))[0]
        order = ok[np.lexsort((ok, d[ok]))][:k]
        cnt[qi] = len(order)
        out["pixel"][qi, : len(order)] = order
        out["dist"][qi, : len(order)] = d[order]
    return out, cnt


def make_case(seed, n_entries=6000, n_queries=3000):
    rng = np.random.default_rng(seed)
    pos = rng.normal(size=(n_entries, 3)).astype(np.float32) * np.float32(2.0)
    pos[: n_entries // 4] = rng.uniform(-0.2, 0.2, (n_entries // 4, 3))  # a dense cluster
    pos[10:20] = pos[0]  # duplicate positions: ties broken by index
    rad = rng.uniform(0.0, 0.4, n_entries).astype(np.float32)
    rad[rng.random(n_entries) < 0.1] = -1.0  # absent entries
    rad[30:40] = 0.0
    entries = np.concatenate([pos, rad[:, None]], axis=1).astype(np.float32)
    queries = np.concatenate([rng.normal(size=(n_queries // 2, 3)) * 2.0,
                              rng.uniform(-0.25, 0.25, (n_queries - n_queries // 2, 3))]).astype(np.float32)
    queries[0] = pos[0]
    return entries, queries


def gpu_search(entries, queries, k, fn="crisb_endpoint_search"):
    lib = _abi.load()
    e = torch.from_numpy(entries).cuda()
    q = torch.from_numpy(queries).cuda()
    out = torch.full((len(queries), k, 2), -7, dtype=torch.int32, device="cuda")
    cnt = torch.full((len(queries),), -7, dtype=torch.int32, device="cuda")
    _abi.check(getattr(lib, fn)(ctypes.c_void_p(e.data_ptr()), len(entries), ctypes.c_void_p(q.data_ptr()),
                                len(queries), k, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr()),
                                None))
    torch.cuda.synchronize()
    return (out.cpu().numpy().reshape(-1).view(_abi.NEIGHBOR_DTYPE).reshape(len(queries), k),
            cnt.cpu().numpy().view(np.uint32))


@pytest.mark.parametrize("k", [1, 8, 31])
def test_endpoint_search_matches_brute_force(cuda_device, k):
    entries, queries = make_case(k)
    got, gc = gpu_search(entries, queries, k)
    ref, rc = brute_force(entries, queries, k)
    assert (gc == rc).all()
    assert got.tobytes() == ref.tobytes()
    assert rc.max() == k and (rc == 0).any()
    assert _abi.load().crisb_endpoint_search_status(None) == _abi.OK


@pytest.mark.parametrize("fn", ["crisb_endpoint_search", "crisb_endpoint_search_noalloc"])
def test_capped_query_reports_device_error(cuda_device, fn):
    """A query that runs out of node visits keeps a partial list and the
    status call reports it (a bounded loop that gives up, not a fault); the
    word is cleared by reading it."""
    lib = _abi.load()
    entries, queries = make_case(7, n_entries=6000, n_queries=500)
    try:
        lib.crisb_endpoint_search_set_visit_cap(3)
        got, gc = gpu_search(entries, queries, 8, fn)
        rc = lib.crisb_endpoint_search_status(None)
        buf = ctypes.create_string_buffer(256)
        lib.crisb_last_error(buf, 256)
    finally:
        lib.crisb_endpoint_search_set_visit_cap(0)
    assert rc == _abi.ERR_DEVICE_FAULT and b"visit cap" in buf.value
    assert lib.crisb_endpoint_search_status(None) == _abi.OK  # read clears it
    ref, refc = brute_force(entries, queries, 8)
    assert (gc <= refc).all() and gc.sum() < refc.sum()
    got2, gc2 = gpu_search(entries, queries, 8, fn)
    assert lib.crisb_endpoint_search_status(None) == _abi.OK
    assert (gc2 == refc).all() and got2.tobytes() == ref.tobytes()


def test_misaligned_outputs_rejected(cuda_device):
    lib = _abi.load()
    e = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    q = torch.zeros((2, 3), dtype=torch.float32, device="cuda")
    out = torch.zeros(64, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(8, dtype=torch.int32, device="cuda")
    for fn in ("crisb_endpoint_search", "crisb_endpoint_search_noalloc"):
        f = getattr(lib, fn)
        rc = f(ctypes.c_void_p(e.data_ptr()), 4, ctypes.c_void_p(q.data_ptr()), 2, 4,
               ctypes.c_void_p(out.data_ptr() + 2), ctypes.c_void_p(cnt.data_ptr()), None)
        assert rc == _abi.ERR_INVALID_ARGUMENT
        rc = f(ctypes.c_void_p(e.data_ptr()), 4, ctypes.c_void_p(q.data_ptr()), 2, 4,
               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(cnt.data_ptr() + 2), None)
        assert rc == _abi.ERR_INVALID_ARGUMENT


def test_endpoint_search_edge_cases(cuda_device):
    lib = _abi.load()
    q = np.zeros((4, 3), np.float32)
    # no entries at all: every count is zero
    got, gc = gpu_search(np.zeros((0, 4), np.float32).reshape(0, 4), q, 4)
    assert (gc == 0).all()
    # a single entry
    e = np.array([[0.0, 0.0, 0.0, 1.0]], np.float32)
    got, gc = gpu_search(e, q, 4)
    assert (gc == 1).all() and (got["pixel"][:, 0] == 0).all()
    # invalid k is rejected without touching the device
    assert lib.crisb_endpoint_search(None, 0, None, 0, 0, None, None, None) == _abi.ERR_INVALID_ARGUMENT
    assert lib.crisb_endpoint_search(None, 0, None, 0, 32, None, None, None) == _abi.ERR_INVALID_ARGUMENT
