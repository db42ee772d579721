"""Tone mapping (src/kernel/tonemap.cu) and headless frame files.

CPU: the oracle's x^(1/2.4) against numpy's float64 power, the oracle's sRGB
bytes against a float64 restatement of the curve away from byte boundaries,
the reference's special-value behaviour, and PNG / PFM round trips.  GPU:
crisb_tonemap_srgb8 bit for bit against the oracle, on byte-boundary inputs,
special values, ragged sizes and a rendered frame."""
import ctypes
import os

import numpy as np
import pytest

import oracle_py as op
from crisoptix_b200 import _abi, image


def _log_uniform(n, seed, lo=-7.0, hi=3.0):
    rng = np.random.default_rng(seed)
    return (10.0 ** rng.uniform(lo, hi, n)).astype(np.float32)


def _boundary_inputs():
    """Linear values whose curve lands on k / 255 for every byte k, and their
    neighbours up to 4 ulps either side: the inputs where a last-bit
    difference in the curve would change the byte."""
    g = np.arange(1, 256, dtype=np.float64) / 255.0
    c = np.where(g <= 0.04045, g / 12.92, ((g + 0.055) / 1.055) ** 2.4).astype(np.float32)
    out = [c]
    up, down = c.copy(), c.copy()
    for _ in range(4):
        up = np.nextafter(up, np.float32(np.inf))
        down = np.nextafter(down, np.float32(0))
        out += [up, down]
    t = np.float32(0.0031308)
    out.append(np.array([t, np.nextafter(t, np.float32(0)), np.nextafter(t, np.float32(1))], np.float32))
    return np.concatenate(out)


SPECIAL = np.array([0.0, -0.0, -1.0, -1e-30, np.nan, np.inf, -np.inf, 1.0, 2.0, 1e6, 1e30, 2e37, 3e37, 3.4e38,
                    1e-45, 1e-38, 0.5, 0.0031308], np.float32)


def test_srgb_root_matches_float64_power():
    x = np.concatenate([_log_uniform(1_000_000, 3, -45, 38), _boundary_inputs(),
                        np.array([1.4e-45, 1.17549435e-38, 1.0, 3.4028235e38], np.float32)])
    got = op.srgb_root(x)
    want = np.power(x.astype(np.float64), 1.0 / 2.4).astype(np.float32)
    bad = np.flatnonzero(got != want)
    # the series is within 1e-14 relative of the power: a float can differ
    # only where the power lies that close to a rounding midpoint
    assert len(bad) <= 2, (x[bad[:5]], got[bad[:5]], want[bad[:5]])
    ulp = np.abs(got[bad].view(np.int32).astype(np.int64) - want[bad].view(np.int32).astype(np.int64))
    assert (ulp <= 1).all()


def test_srgb_root_special_values():
    got = op.srgb_root(np.array([0.0, -0.0, np.inf, -1.0, np.nan, -np.inf], np.float32))
    assert got[0] == 0 and got[1] == 0 and got[2] == np.inf
    assert np.isnan(got[3:]).all()


def _curve64(c):
    c = c.astype(np.float64)
    with np.errstate(invalid="ignore"):
        g = np.where(c < 0.0031308, 12.92 * c, 1.055 * np.power(np.maximum(c, 0), 1 / 2.4) - 0.055)
    return np.clip(g, 0, 1) * 255.0


def test_tonemap_oracle_against_float64_curve():
    x = np.concatenate([_log_uniform(300_000, 4), -_log_uniform(1000, 5), _boundary_inputs()])
    x = x[: len(x) // 3 * 3].reshape(-1, 3)
    got = op.tonemap_srgb8(x).astype(np.int64)
    exact = _curve64(x)
    want = np.floor(exact).astype(np.int64)
    frac = exact - np.floor(exact)
    far = (frac > 1e-4) & (frac < 1 - 1e-4)
    assert (got[far] == want[far]).all()
    assert np.abs(got - want).max() <= 1
    inside = (exact > 0) & (exact < 255)
    assert far[inside].mean() > 0.95  # the boundary inputs are about 2% of the set


def test_tonemap_reference_special_values():
    """The reference blends both branches (if_false * (1 - cond) + if_true *
    cond) and clamps with a NaN-preserving clamp: negative channels (pow gives
    NaN), NaN, +inf and values whose 12.92 c overflows all come out 0."""
    x = np.resize(SPECIAL, (len(SPECIAL) + 2) // 3 * 3).reshape(-1, 3)
    got = dict(zip(x.ravel().tolist()[:len(SPECIAL)], op.tonemap_srgb8(x).ravel().tolist()))
    assert got[0.0] == 0 and got[-1.0] == 0 and got[float(np.float32(-1e-30))] == 0
    assert got[float("inf")] == 0 and got[float("-inf")] == 0
    assert got[float(np.float32(3e37))] == 0 and got[float(np.float32(3.4e38))] == 0  # 12.92 c = inf
    assert got[float(np.float32(2e37))] == 255 and got[2.0] == 255 and got[1e6] == 255
    # c = 1: 1.055f - 0.055f rounds to 0.99999994f in float, so 254
    assert got[1.0] == 254
    assert got[0.5] == 187
    assert op.tonemap_srgb8(np.array([[np.nan, 1.0, 0.5]], np.float32)).tolist() == [[0, 254, 187]]


def test_png_round_trip_and_orientation(tmp_path):
    rng = np.random.default_rng(6)
    a = rng.integers(0, 256, (37, 53, 3), dtype=np.uint8)
    p = str(tmp_path / "f.png")
    image.write_png(p, a)
    data = open(p, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n" and data[12:16] == b"IHDR"
    back = image.decode_png(data)
    assert (back == a).all()  # row 0 of a frame is the top row of the file
    assert (image.decode_png(image.encode_png(a, bottom_up=True)) == a[::-1]).all()
    with pytest.raises(ValueError):
        image.encode_png(a.astype(np.float32))


def test_pfm_round_trip(tmp_path):
    a = _log_uniform(24 * 17 * 3, 8).reshape(17, 24, 3)
    p = str(tmp_path / "f.pfm")
    image.write_pfm(p, a)
    assert open(p, "rb").read(3) == b"PF\n"
    assert os.path.getsize(p) == len(b"PF\n24 17\n-1.0\n") + a.nbytes
    assert (image.read_pfm(p) == a).all()
    raw = np.frombuffer(open(p, "rb").read()[len(b"PF\n24 17\n-1.0\n"):], "<f4").reshape(17, 24, 3)
    assert (raw[0] == a[-1]).all()  # PFM stores the bottom row first


def _thresholds():
    t = np.zeros(256, np.float32)
    c_max = ctypes.c_float()
    assert _abi.load().crisb_srgb8_thresholds(t.ctypes.data, ctypes.byref(c_max)) == 0
    return t, np.float32(c_max.value)


def _lookup(t, c_max, x):
    """The kernel's rule: count of thresholds k >= 1 at or below c on
    [0, c_max], 0 elsewhere."""
    x = np.asarray(x, np.float32)
    with np.errstate(invalid="ignore"):
        inside = (x >= 0) & (x <= c_max)
    return np.where(inside, np.searchsorted(t[1:], x, side="right"), 0).astype(np.uint8)


def test_kernel_step_table_is_the_oracle_curve():
    """The library's host-built step table against the oracle's formula: each
    threshold is a step of the oracle's bytes (byte >= k there, < k one float
    below), the bytes never decrease between the first step and 2.0 (every
    float checked), and the table rule reproduces the formula elsewhere."""
    t, c_max = _thresholds()
    assert t[0] == 0 and (np.diff(t) >= 0).all()
    k = np.arange(1, 256)
    at = op.tonemap_srgb8(t[1:].reshape(-1, 3)).ravel()
    below = op.tonemap_srgb8(np.nextafter(t[1:], np.float32(0)).reshape(-1, 3)).ravel()
    assert (at >= k).all() and (below < k).all()
    with np.errstate(over="ignore"):
        assert np.isfinite(np.float32(12.92) * c_max)
        assert np.isinf(np.float32(12.92) * np.nextafter(c_max, np.float32(np.inf)))
    assert op.srgb8_first_decrease(float(t[1]) / 2, 2.0) == 0
    x = np.concatenate([_log_uniform(600_000, 12, -9, 38), -_log_uniform(3000, 13), _boundary_inputs(), SPECIAL,
                        np.array([c_max, np.nextafter(c_max, np.float32(np.inf))], np.float32)])
    x = np.resize(x, (len(x) + 2) // 3 * 3).reshape(-1, 3)
    assert (_lookup(t, c_max, x) == op.tonemap_srgb8(x)).all()
    low = _log_uniform(30_000, 14, -44, np.log10(float(t[1]) / 2)).reshape(-1, 3)
    assert (op.tonemap_srgb8(low) == 0).all()


def test_tonemap_entry_point_declared():
    assert "crisb_tonemap_srgb8" in _abi.ENTRY_POINTS
    fn = getattr(_abi.load(), "crisb_tonemap_srgb8")
    assert fn.restype is ctypes.c_int32


def _gpu_tonemap(x):
    import torch

    d = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    out = image.tonemap(d)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
def test_tonemap_gpu_bit_parity(cuda_device):
    t, c_max = _thresholds()
    steps = np.concatenate([t[1:], np.nextafter(t[1:], np.float32(0)), [c_max, np.nextafter(c_max, np.inf)]])
    x = np.concatenate([_log_uniform(3 * 400_000, 9, -8, 4), -_log_uniform(3000, 10), _boundary_inputs(),
                        SPECIAL, steps.astype(np.float32)])
    x = np.resize(x, (len(x) + 2) // 3 * 3).reshape(-1, 3)
    assert (_gpu_tonemap(x) == op.tonemap_srgb8(x)).all()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 255, 256, 257, 1023, 148 * 256 + 7])
def test_tonemap_gpu_ragged_sizes(cuda_device, n):
    x = _log_uniform(3 * n, n, -5, 1).reshape(n, 3)
    assert (_gpu_tonemap(x) == op.tonemap_srgb8(x)).all()


@pytest.mark.gpu
def test_tonemap_gpu_unaligned_pointers(cuda_device):
    """Pointers off the 16-byte / 4-byte alignment of the four-pixel path take
    the pixel-by-pixel path."""
    import torch

    n = 1001
    x = _log_uniform(3 * n, 15, -5, 1)
    src = torch.zeros(3 * n + 1, dtype=torch.float32, device="cuda")
    src[1:] = torch.from_numpy(x).cuda()
    dst = torch.zeros(3 * n + 1, dtype=torch.uint8, device="cuda")
    assert _abi.load().crisb_tonemap_srgb8(src.data_ptr() + 4, dst.data_ptr() + 1, n, 0) == 0
    torch.cuda.synchronize()
    got = dst.cpu().numpy()
    assert got[0] == 0 and (got[1:] == op.tonemap_srgb8(x.reshape(n, 3)).ravel()).all()


@pytest.mark.gpu
def test_tonemap_gpu_empty_and_null(cuda_device):
    import torch

    lib = _abi.load()
    buf = torch.zeros(3, device="cuda")
    assert lib.crisb_tonemap_srgb8(buf.data_ptr(), buf.data_ptr(), 0, 0) == 0
    assert lib.crisb_tonemap_srgb8(None, buf.data_ptr(), 1, 0) == _abi.ERR_INVALID_ARGUMENT
    assert image.tonemap(torch.zeros((0, 3), device="cuda")).shape == (0, 3)


@pytest.mark.gpu
def test_tonemap_rendered_frame(cuda_device, tmp_path):
    import torch

    from crisoptix_b200 import Renderer, Scene, scenes
    from helpers import scene_size_of, small_config_params

    desc, cam = scenes.cornell_box()
    W, H = 64, 48
    r = Renderer(W, H, Scene(desc), small_config_params(scene_size_of(desc)))
    hdr = torch.zeros((H, W, 3), dtype=torch.float32, device="cuda")
    for _ in range(2):
        r.launch_frame(cam, hdr.data_ptr())
    torch.cuda.synchronize()
    p = str(tmp_path / "frame.png")
    srgb = image.save_frame(p, hdr)
    assert (srgb == op.tonemap_srgb8(hdr.cpu().numpy())).all()
    assert (image.decode_png(open(p, "rb").read()) == srgb).all()
    assert srgb.mean() > 20


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("rtype", [_abi.CONDITIONAL_RESTIR, _abi.RESTIR_PT, _abi.PATH_TRACER])
def test_frame_srgb_output(cuda_device, graph, rtype):
    """The frame loop with the sRGB epilogue (LaunchFrame then ToneMapping):
    float frame and bytes both bit-exact with the oracle, every frame, in and
    out of the frame graph; turning the output off stops the writes."""
    import torch

    from crisoptix_b200 import Renderer, Scene, scenes
    from helpers import scene_size_of, small_config_params

    desc, cam = scenes.cornell_box()
    W, H = 48, 40
    p = small_config_params(scene_size_of(desc), renderer_type=rtype)
    sc = Scene(desc)
    o = op.Oracle.from_scene(desc, W, H, p, triangles=sc.read_triangles())
    r = Renderer(W, H, sc, p)
    r.set_graph(graph)
    hdr = torch.zeros(H * W * 3, dtype=torch.float32, device="cuda")
    srgb = torch.zeros(H * W * 3, dtype=torch.uint8, device="cuda")
    r.set_srgb_output(srgb.data_ptr())
    out_h = np.zeros((H, W, 3), np.float32)
    for _ in range(3):
        r.launch_frame(cam, hdr.data_ptr())
        o.render_frame(cam, out_h)
        torch.cuda.synchronize()
        r.check_device_errors()
        assert hdr.cpu().numpy().tobytes() == out_h.tobytes()
        assert (srgb.cpu().numpy() == op.tonemap_srgb8(out_h).ravel()).all()
    assert int(srgb.sum()) > 0
    r.set_srgb_output(0)
    srgb.zero_()
    r.launch_frame(cam, hdr.data_ptr())
    torch.cuda.synchronize()
    assert int(srgb.sum()) == 0
