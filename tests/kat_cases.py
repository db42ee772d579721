"""Inputs and packing for the known-answer tests of oracle/kat.h.

The same seeded inputs drive the reference's compiled code (fixture
generation), the oracle (CPU suite) and the CUDA device functions (GPU
suite).  Records are arrays of 32-bit words; 64-bit values are two words,
low word first.
"""
from __future__ import annotations

import ctypes

import numpy as np

FUNCTIONS = {"tea64": 1, "pcg_seed": 2, "pcg_draws": 3, "luminance": 4, "mis_canon": 5, "mis_neigh": 6,
             "select_neighbor": 7, "jacobian": 8, "reservoir": 9, "ggx": 10, "camera_ray": 11}
RES_STEPS = 8
IN_WORDS = [0, 2, 4, 4, 3, 10, 10, 6, 12, 4 + 2 + 3 + 5 * RES_STEPS, 8, 14]
OUT_WORDS = [0, 2, 4, 6, 1, 1, 1, 4, 1, 3 * RES_STEPS + 4, 5, 3]
N_CASES = 1024

# output words that hold floats, per function (any NaN equals any NaN there:
# NaN payloads differ between x86 and the GPU, and no function here defines
# one)
FLOAT_WORDS = {1: [], 2: [], 3: [1], 4: [0], 5: [0], 6: [0], 7: [], 8: [0],
               9: [w for s in range(RES_STEPS) for w in (3 * s + 1, 3 * s + 2)] + [3 * RES_STEPS + 1],
               10: [0, 1, 2, 3, 4], 11: [0, 1, 2]}


def same_nan(fn: int, got: np.ndarray, want: np.ndarray) -> np.ndarray:
    """got and want with the NaNs of float words made identical"""
    got, want = got.copy(), want.copy()
    for w in FLOAT_WORDS[fn]:
        both = np.isnan(got[:, w].view(np.float32)) & np.isnan(want[:, w].view(np.float32))
        got[both, w] = want[both, w]
    return got

EMITTER_DTYPE = np.dtype([("color", np.float32, 3), ("first_face", np.uint32), ("num_faces", np.uint32)])


def _u64_words(v: np.ndarray) -> np.ndarray:
    v = np.asarray(v, np.uint64)
    return np.stack([(v & np.uint64(0xFFFFFFFF)).astype(np.uint32), (v >> np.uint64(32)).astype(np.uint32)], -1)


def _f(a) -> np.ndarray:
    return np.asarray(a, np.float32).view(np.uint32)


def _special(rng, n, scale=1.0):
    """float32 values with the special cases mixed in"""
    v = (rng.standard_normal(n) * scale).astype(np.float32)
    k = rng.integers(0, 10, n)
    v[k == 0] = 0.0
    v[k == 1] = np.float32(np.nan)
    v[k == 2] = np.float32(np.inf) * np.sign(rng.standard_normal((k == 2).sum())).astype(np.float32)
    v[k == 3] = np.float32(1e-40)  # subnormal
    v[k == 4] = np.float32(3e38)
    return v


def _rgb(rng, n, zero_frac=0.15):
    c = np.exp(rng.normal(0.0, 2.0, (n, 3))).astype(np.float32)
    c[rng.random(n) < zero_frac] = 0.0
    return c


def _states(rng, n):
    st = rng.integers(0, 2 ** 63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    inc = (rng.integers(0, 2 ** 63, n, dtype=np.uint64) << np.uint64(1)) | np.uint64(1)
    inc[: n // 2] = np.uint64((0xda3e39cb94b95bdb * 2 + 1) & 0xFFFFFFFFFFFFFFFF)  # the default stream
    return np.concatenate([_u64_words(st), _u64_words(inc)], -1)


def inputs(fn: int, seed: int, n: int = N_CASES) -> np.ndarray:
    rng = np.random.default_rng(1000 + seed)
    if fn == 1:  # TEA64
        w = rng.integers(0, 2 ** 32, (n, 2), dtype=np.uint64).astype(np.uint32)
        w[:8] = [[0, 0], [0xFFFFFFFF, 0xFFFFFFFF], [0, 1], [1, 0], [1920 * 1080 - 1, 12345], [5, 0xDEADBEEF],
                 [65535, 7], [2 ** 31, 2 ** 31]]
        return w
    if fn == 2:  # PCG seed
        a = rng.integers(0, 2 ** 63, (n, 2), dtype=np.uint64)
        a[n // 2:, 1] = np.uint64(0xda3e39cb94b95bdb)  # the default stream, as the reference seeds
        a[:4] = [[0, 0], [42, 54], [0, 1], [12345, 0]]
        return np.concatenate([_u64_words(a[:, 0]), _u64_words(a[:, 1])], -1)
    if fn == 3:
        return _states(rng, n)
    if fn == 4:
        return _f(np.stack([_special(rng, n), _special(rng, n), _special(rng, n)], -1))
    if fn in (5, 6):
        a, b = _rgb(rng, n), _rgb(rng, n)
        jac = np.exp(rng.normal(0.0, 1.5, n)).astype(np.float32)
        jac[rng.random(n) < 0.1] = 0.0
        jac[rng.random(n) < 0.02] = np.float32(np.inf)
        K = rng.integers(1, 17, n).astype(np.float32)
        cm = rng.choice(np.array([0.0, 1.0, 2.0, 20.0, 50.0], np.float32), n)
        nm = rng.uniform(0.0, 50.0, n).astype(np.float32)
        nm[rng.random(n) < 0.1] = 0.0
        return _f(np.concatenate([a, b, jac[:, None], K[:, None], cm[:, None], nm[:, None]], -1))
    if fn == 7:
        px = rng.integers(0, 2000, n).astype(np.uint32)
        py = rng.integers(0, 1200, n).astype(np.uint32)
        px[:16] = np.arange(16) % 11  # near the origin: the window wraps below zero
        py[:16] = np.arange(16) % 7
        px[16:20] = 0xFFFFFFF5
        return np.concatenate([px[:, None], py[:, None], _states(rng, n)], -1)
    if fn == 8:
        p = rng.normal(0.0, 2.0, (n, 4, 3)).astype(np.float32)
        nrm = p[:, 3] / np.linalg.norm(p[:, 3], axis=1, keepdims=True)
        p[:, 3] = nrm
        p[:8, 1] = p[:8, 2]      # new point on the target: division by zero
        p[8:16, 0] = p[8:16, 2]  # old point on the target: NaN
        p[16:24, 3] = 0.0        # zero normal
        return _f(p.reshape(n, 12))
    if fn == 9:
        w = np.exp(rng.normal(0.0, 2.0, (n, RES_STEPS))).astype(np.float32)
        k = rng.integers(0, 12, (n, RES_STEPS))
        w[k == 0] = 0.0
        w[k == 1] = np.float32(np.nan)
        w[k == 2] = np.float32(np.inf)
        w[k == 3] = np.float32(-np.inf)
        w[k == 4] = -w[k == 4]
        conf = rng.choice(np.array([0.0, 1.0, 2.0, 7.0, 50.0], np.float32), (n, RES_STEPS))
        f = _rgb(rng, n * RES_STEPS).reshape(n, RES_STEPS, 3)
        cand = np.concatenate([w[..., None], conf[..., None], f], -1).reshape(n, 5 * RES_STEPS)
        w0 = np.where(rng.random(n) < 0.5, 0.0, np.exp(rng.normal(0, 2, n))).astype(np.float32)
        c0 = rng.choice(np.array([0.0, 1.0, 49.5], np.float32), n)
        f0 = _rgb(rng, n, zero_frac=0.3)
        return np.concatenate([_states(rng, n), _f(w0)[:, None], _f(c0)[:, None], _f(f0), _f(cand)], -1)
    if fn == 10:
        ndoth = rng.uniform(0.0, 1.0, n)
        ndotl = rng.uniform(1e-4, 1.0, n)
        ndotv = rng.uniform(1e-4, 1.0, n)
        rough = rng.uniform(0.05, 1.0, n)
        vdoth = rng.uniform(0.0, 1.0, n)
        vdoth[:32] = rng.uniform(1.0, 1.5, 32)  # 1 - VdotH below zero: clamped
        f0 = rng.uniform(0.0, 1.0, (n, 3))
        f0[:16] = 0.04
        ndoth[32:40] = 1.0
        rough[40:48] = 1.0
        return _f(np.concatenate([np.stack([ndoth, ndotl, ndotv, rough, vdoth], -1), f0], -1))
    if fn == 11:
        pos = rng.normal(0.0, 5.0, (n, 3))
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        tan_half = np.tan(0.5 * rng.uniform(0.3, 1.8, n))
        aspect = rng.uniform(0.5, 2.5, n)
        U = q[0][None] * (tan_half * aspect)[:, None]
        V = -q[1][None] * tan_half[:, None]
        W = np.repeat(-q[2][None], n, 0)
        vp = rng.uniform(-1.0, 1.0, (n, 2))
        return _f(np.concatenate([pos, U, V, W, vp], -1))
    raise ValueError(fn)


def run(call, fn: int, inp: np.ndarray) -> np.ndarray:
    """call(fn, in_ptr, n, out_ptr) -> status; returns the packed outputs"""
    inp = np.ascontiguousarray(inp, np.uint32)
    n = inp.shape[0]
    assert inp.shape[1] == IN_WORDS[fn]
    out = np.zeros((n, OUT_WORDS[fn]), np.uint32)
    rc = call(fn, inp.ctypes.data_as(ctypes.c_void_p), n, out.ctypes.data_as(ctypes.c_void_p))
    assert rc == 0, rc
    return out


def emitter_case(seed: int, n_draws: int = 2048):
    rng = np.random.default_rng(seed)
    counts = np.array([1, 3, 7, 2, 5], np.uint32)
    ems = np.zeros(len(counts), EMITTER_DTYPE)
    ems["num_faces"] = counts
    ems["first_face"] = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    ems["color"] = rng.uniform(1.0, 20.0, (len(counts), 3))
    faces = rng.normal(0.0, 3.0, (int(counts.sum()), 9)).astype(np.float32)
    st = rng.integers(0, 2 ** 63, n_draws, dtype=np.uint64)
    inc = (rng.integers(0, 2 ** 62, n_draws, dtype=np.uint64) << np.uint64(1)) | np.uint64(1)
    states = np.stack([st, inc], -1)
    return ems, faces, states


def run_emitter(fn, ems, faces, states):
    ems = np.ascontiguousarray(ems)
    faces = np.ascontiguousarray(faces, np.float32)
    states = np.ascontiguousarray(states, np.uint64)
    n = len(states)
    out = np.zeros((n, 6), np.float32)
    st = np.zeros(n, np.uint64)
    vp = ctypes.c_void_p
    rc = fn(ems.ctypes.data_as(vp), len(ems), faces.ctypes.data_as(vp), states.ctypes.data_as(vp), n,
            out.ctypes.data_as(vp), st.ctypes.data_as(vp))
    assert rc == 0, rc
    return out, st
