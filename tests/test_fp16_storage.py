"""FP16 reservoir storage: the oracle's binary16 and octahedral codecs on CPU
(against numpy and by round trip), and on the GPU bit parity of the packed
reservoirs and the image with the oracle in the same storage mode."""
import numpy as np
import pytest

import oracle_py as op
from crisoptix_b200 import _abi


def test_half_matches_numpy_round_to_nearest_even():
    rng = np.random.default_rng(5)
    vals = [rng.standard_normal(20000).astype(np.float32) * s for s in (1e-7, 1e-5, 1e-3, 1.0, 100.0, 3e4)]
    x = np.concatenate(vals + [np.array([0.0, -0.0, 65504.0, -65504.0, 6.1e-5, 5.96e-8, 2.98e-8], np.float32)])
    # exact ties between neighbouring binary16 values
    h = np.arange(1, 0x7bff, 37, dtype=np.uint16).view(np.float16).astype(np.float32)
    h_next = (np.arange(1, 0x7bff, 37, dtype=np.uint16) + 1).view(np.float16).astype(np.float32)
    ties = ((h.astype(np.float64) + h_next.astype(np.float64)) / 2).astype(np.float32)
    x = np.concatenate([x, ties, -ties])
    bits, back = op.half(x)
    want = np.clip(x, -65504.0, 65504.0).astype(np.float16)  # the storage rule saturates
    assert (bits == want.view(np.uint16)).all()
    assert (back == want.astype(np.float32)).all()


def test_half_saturates_and_zeroes_nan():
    bits, back = op.half(np.array([1e6, -1e6, np.inf, -np.inf, np.nan, 65520.0], np.float32))
    assert list(back) == [65504.0, -65504.0, 65504.0, -65504.0, 0.0, 65504.0]


def _unit(n, seed):
    d = np.random.default_rng(seed).standard_normal((n, 3)).astype(np.float32)
    return (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)


def test_octahedral_round_trip_error():
    d = _unit(50000, 7)
    axes = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float32)
    d = np.concatenate([d, axes])
    codes, dec = op.oct(d)
    chord = np.linalg.norm(dec.astype(np.float64) - d, axis=1)  # ~ angle in radians
    assert chord.max() < 1e-4
    assert np.abs(np.linalg.norm(dec, axis=1) - 1).max() < 1e-6
    codes0, dec0 = op.oct(np.zeros((1, 3), np.float32))
    assert codes0[0] == _abi.OCT_ZERO and (dec0 == 0).all()


def test_octahedral_codes_are_stable_under_reencoding():
    """Storing a loaded direction again must not move its code (the library
    re-stores loaded reservoirs; the oracle quantises once per pass)."""
    rng = np.random.default_rng(11)
    q = rng.integers(-32767, 32768, size=(200000, 2))
    edge = np.array([[x, y] for x in (-32767, -1, 0, 1, 32767) for y in (-32767, -1, 0, 1, 32767)])
    q = np.concatenate([q, edge])
    codes = ((q[:, 0] & 0xFFFF) | ((q[:, 1] & 0xFFFF) << 16)).astype(np.uint32)
    # decode through the oracle by encoding the decoded vectors twice
    _, dec = op.oct(_decode_py(codes))
    codes2, _ = op.oct(dec)
    codes3, _ = op.oct(_decode_py(codes2))
    assert (codes3 == codes2).all()
    _, d1 = op.oct(dec)
    _, d2 = op.oct(_decode_py(codes2))
    assert (d1 == d2).all()


def test_octahedral_codes_on_the_fold_edge_are_stable():
    """Every code with a coordinate on the fold's edge or next to it, and
    every code of a coarse grid, re-encodes to a stable code; and a fresh
    direction's code survives decode + re-encode.  The fold edge (|x| or
    |y| = 32767) decodes to a signed zero in the other coordinate: it once
    flipped sign on re-encoding (the sign test was v >= 0), which made 43 of
    the 2 M primary-hit codes of a 1080p frame differ between a record stored
    once and one stored twice."""
    import ctypes

    edge = np.array([-32767, -32766, -32765, -2, -1, 0, 1, 2, 32765, 32766, 32767])
    full = np.arange(-32767, 32768)
    grid = np.arange(-32767, 32768, 97)
    pairs = [np.stack(np.meshgrid(a, b), -1).reshape(-1, 2) for a, b in ((edge, full), (full, edge), (grid, grid))]
    q = np.concatenate(pairs)
    codes = ((q[:, 0] & 0xFFFF) | ((q[:, 1] & 0xFFFF) << 16)).astype(np.uint32)
    lib = op.load()
    assert lib.oracle_oct_unstable(codes.ctypes.data_as(ctypes.c_void_p), len(codes)) == 0
    # fresh directions, signed zeros and axis-aligned ones included
    d = _unit(200000, 13)
    d[:1000, 0] = -0.0
    d[1000:2000, 1] = -0.0
    d[2000:2006] = [[0, 0, -1], [-0.0, 0, -1], [0, -0.0, -1], [-0.0, -0.0, -1], [1, 0, 0], [-1, -0.0, 0]]
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    c1, dec = op.oct(d)
    c2, _ = op.oct(dec)
    assert (c1 == c2).all()


def _decode_py(codes):
    """float64 decode of octahedral codes, used only to produce directions
    near each code's centre for the oracle to encode."""
    x = (codes & 0xFFFF).astype(np.uint16).view(np.int16).astype(np.float64) / 32767.0
    y = (codes >> 16).astype(np.uint16).view(np.int16).astype(np.float64) / 32767.0
    z = 1 - np.abs(x) - np.abs(y)
    neg = z < 0
    tx = (1 - np.abs(y)) * np.where(x >= 0, 1, -1)
    ty = (1 - np.abs(x)) * np.where(y >= 0, 1, -1)
    x = np.where(neg, tx, x)
    y = np.where(neg, ty, y)
    v = np.stack([x, y, z], axis=1)
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["cornell", "spheres"])
def test_fp16_storage_bit_parity(cuda_device, which):
    from crisoptix_b200 import scenes
    from helpers import large_config_params, orbit, scene_size_of, small_config_params, small_sphere_room, static
    from test_parity_gpu import run_parity

    if which == "cornell":
        desc, cam = scenes.cornell_box()
        p = small_config_params(scene_size_of(desc), storage=_abi.STORAGE_FP16)
        run_parity(desc, cam, p, 48, 40, 4, static)
    else:
        desc, cam = small_sphere_room()
        p = large_config_params(scene_size_of(desc), gather_radius=0.3, storage=_abi.STORAGE_FP16)
        run_parity(desc, cam, p, 64, 48, 4, lambda c, f: orbit(c, f, 120))


@pytest.mark.gpu
def test_fp16_storage_restir_pt(cuda_device):
    from crisoptix_b200 import scenes
    from helpers import make_params, scene_size_of, static
    from test_parity_gpu import run_parity

    desc, cam = scenes.cornell_box()
    p = make_params(scene_size_of(desc), renderer_type=_abi.RESTIR_PT, max_path_len=5, prefix_enable_spatial=1,
                    prefix_spatial_count=3, prefix_spatial_rounds=2, storage=_abi.STORAGE_FP16)
    run_parity(desc, cam, p, 40, 40, 3, static)
