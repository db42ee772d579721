"""Known-answer and accuracy tests of the oracle's building blocks (CPU)."""
import math

import numpy as np

import oracle_py as op
from crisoptix_b200 import scenes


def test_pcg32_published_demo_sequence():
    # pcg32 demo (O'Neill, pcg-c-basic): seed 42, sequence 54 -- the generator
    # of include/util/random.h:45-119 is this PCG32 (XSH RR, 64-bit state).
    out = op.pcg32(42, 54, 6)
    assert [hex(int(v)) for v in out] == ["0xa15c02b7", "0x7b47f409", "0xba1d3330", "0x83d2f293", "0xbfa4784b",
                                          "0xcbed606e"]


def _tea64_py(v0, v1):
    s0 = 0
    m = 0xFFFFFFFF
    for _ in range(4):
        s0 = (s0 + 0x9E3779B9) & m
        v0 = (v0 + ((((v1 << 4) + 0xA341316C) & m) ^ ((v1 + s0) & m) ^ (((v1 >> 5) + 0xC8013EA4) & m))) & m
        v1 = (v1 + ((((v0 << 4) + 0xAD90777D) & m) ^ ((v0 + s0) & m) ^ (((v0 >> 5) + 0x7E95761E) & m))) & m
    return v0 | (v1 << 32)


def test_tea64_matches_independent_python():
    rng = np.random.default_rng(0)
    for a, b in rng.integers(0, 2**32, (64, 2), dtype=np.uint64):
        assert op.tea64(int(a), int(b)) == _tea64_py(int(a), int(b))


def test_pcg32_default_stream_seeding_matches_python():
    mult, inc = 0x5851F42D4C957F2D, ((0xDA3E39CB94B95BDB << 1) | 1) & (2**64 - 1)
    m64 = 2**64 - 1

    def step(state):
        old = state
        state = (old * mult + inc) & m64
        xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return state, ((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF

    seed = 0x1234_5678_9ABC_DEF0
    st, _ = step(0)
    st = (st + seed) & m64
    st, _ = step(st)
    ref = []
    for _ in range(8):
        st, v = step(st)
        ref.append(v)
    assert list(op.pcg32(seed, 0xDA3E39CB94B95BDB, 8)) == ref


def test_sincos_error_bound():
    phi = (np.arange(1 << 18, dtype=np.float64) / (1 << 18) * 2 * math.pi).astype(np.float32)
    s, c = op.sincos(phi)
    ph = phi.astype(np.float64)
    assert np.abs(s - np.sin(ph)).max() < 1.5e-7
    assert np.abs(c - np.cos(ph)).max() < 1.5e-7


def test_camera_basis_matches_lookat_inverse():
    cam = scenes.Camera((1.0, 2.0, 3.0), (0.3, -0.2, -0.93), (0.0, 1.0, 0.0), 1.5, math.radians(50))
    d = op.camera_data(cam).astype(np.float64)
    f = np.asarray(cam.view_dir) / np.linalg.norm(cam.view_dir)
    s = np.cross(f, cam.up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    t = math.tan(0.5 * cam.fov)
    np.testing.assert_allclose(d[1], s * t * cam.aspect, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(d[2], -u * t, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(d[3], f, rtol=1e-5, atol=1e-6)


def test_frame_random_is_seeded_and_per_frame():
    a = [op.frame_random(3, i) for i in range(8)]
    assert a == [op.frame_random(3, i) for i in range(8)]
    assert len(set(a)) == 8
    assert op.frame_random(4, 0) != a[0]
