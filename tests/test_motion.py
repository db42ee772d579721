"""Temporal reprojection (prevPixelCoord, shader/prefix_gen_temp_reuse.cu:130-136).

CPU: the oracle's three modes -- zero motion vectors reproduce the reference's
own prevPixelCoord = pixelCoord bit for bit; the reprojected previous pixel is
the pixel itself for a still camera and follows a float64 projection for a
moving one; the conversion of out-of-range vectors.  GPU: the library
against the oracle in every mode, FP32 and FP16 storage, with and without the
frame graph."""
import numpy as np
import pytest

import oracle_py as op
from crisoptix_b200 import _abi, scenes
from helpers import orbit, scene_size_of, small_config_params, static

W, H = 48, 40
ALL_BUFS = [_abi.BUF_PREFIX_RES_FRONT, _abi.BUF_PREFIX_RES_BACK, _abi.BUF_CANON_PREFIX, _abi.BUF_SUFFIX_RES_FRONT,
            _abi.BUF_CANON_SUFFIX, _abi.BUF_GBUFFER, _abi.BUF_NEIGHBORS, _abi.BUF_NEIGHBOR_COUNT]


def _oracle(mode, storage=_abi.STORAGE_FP32, **kw):
    desc, cam = scenes.cornell_box()
    p = small_config_params(scene_size_of(desc), motion_mode=mode, storage=storage, **kw)
    return op.Oracle.from_scene(desc, W, H, p), cam


def _frames(o, cam, cam_fn, n):
    out = np.zeros((H, W, 3), np.float32)
    states = []
    for f in range(n):
        o.render_frame(cam_fn(cam, f), out)
        states.append([out.copy()] + [o.dump(b) for b in ALL_BUFS])
    return states


def _prev_xy(o):
    g = o.dump(_abi.BUF_GBUFFER)
    return g["prev_xy"].astype(np.uint32)


def test_zero_motion_vectors_match_the_reference_mode():
    a, cam = _oracle(_abi.MOTION_NONE)
    b, _ = _oracle(_abi.MOTION_VECTORS)
    b.set_motion_vectors(np.zeros((H, W, 2), np.float32))
    sa, sb = _frames(a, cam, lambda c, f: orbit(c, f, 30), 3), _frames(b, cam, lambda c, f: orbit(c, f, 30), 3)
    for fa, fb in zip(sa, sb):
        for x, y in zip(fa, fb):
            assert x.tobytes() == y.tobytes()


def test_motion_vector_conversion():
    """uvec2(pixel + 0.5 + v) with the GPU's saturating conversion: negative
    and NaN components clamp to 0, components past the image make the pixel
    invalid, which the G-buffer stores as 0xffffffff."""
    o, cam = _oracle(_abi.MOTION_VECTORS)
    mv = np.zeros((H, W, 2), np.float32)
    mv[0, 0] = (3.2, 1.7)          # -> (3, 2)
    mv[0, 1] = (-5.0, 0.0)         # x: 1.5 - 5 < 0 -> 0
    mv[0, 2] = (np.nan, 2.0)       # x: NaN -> 0
    mv[0, 3] = (W + 1.0, 0.0)      # off the right edge -> none
    mv[0, 4] = (0.0, 1e30)         # far below -> none
    mv[0, 5] = (-0.6, 0.0)         # 5.5 - 0.6 = 4.9 -> 4
    o.set_motion_vectors(mv)
    out = np.zeros((H, W, 3), np.float32)
    o.render_frame(cam, out)
    pxy = _prev_xy(o)
    assert pxy[0] == 3 | (2 << 16)
    assert pxy[1] == 0 and pxy[2] == 0 | (2 << 16)
    assert pxy[3] == 0xFFFFFFFF and pxy[4] == 0xFFFFFFFF
    assert pxy[5] == 4
    assert pxy[6] == 6  # zero vector: the pixel itself
    o.set_motion_vectors(None)
    with pytest.raises(ValueError):
        o.render_frame(cam, out)


def test_reprojection_still_camera_is_the_pixel_itself():
    o, cam = _oracle(_abi.MOTION_REPROJECT)
    out = np.zeros((H, W, 3), np.float32)
    o.render_frame(cam, out)
    assert (_prev_xy(o) == 0xFFFFFFFF).all()  # no previous camera yet
    o.render_frame(static(cam, 1), out)
    pxy = _prev_xy(o)
    valid = o.dump(_abi.BUF_GBUFFER)["flags"] & 1 == 1
    own = (np.arange(W * H) % W) | ((np.arange(W * H) // W) << 16)
    assert valid.mean() > 0.9
    # the jittered primary hit lies in the pixel's own footprint; rounding
    # can move it over an edge only for hits within an ulp of the border
    assert (pxy[valid] == own[valid]).mean() > 0.995
    assert (pxy[~valid] == 0xFFFFFFFF).all()


def test_reprojection_follows_the_moving_camera():
    """Each pixel with a valid canonical prefix holds the float64 projection of
    its primary hit through the previous camera (to within the rounding of the
    float arithmetic at footprint borders); the others have none."""
    from crisoptix_b200 import camera_data

    o, cam = _oracle(_abi.MOTION_REPROJECT)
    out = np.zeros((H, W, 3), np.float32)
    c0, c1 = orbit(cam, 0, 40), orbit(cam, 1, 40)
    o.render_frame(c0, out)
    o.render_frame(c1, out)
    pxy = _prev_xy(o)
    canon = o.dump(_abi.BUF_CANON_PREFIX)
    pos, _, _ = scenes.cornell_box()[0].flatten()
    pos = pos.reshape(-1, 3, 3).astype(np.float64)
    prim = canon["primary"]["prim"]
    ok = (prim != 0xFFFFFFFF) & ((canon["flags"] >> 16) & 1 == 1)  # a valid canonical prefix
    bary = canon["primary"]["bary"].astype(np.float64)
    tri = pos[np.where(ok, prim, 0)]
    p = (1 - bary[:, :1] - bary[:, 1:]) * tri[:, 0] + bary[:, :1] * tri[:, 1] + bary[:, 1:] * tri[:, 2]
    d = camera_data(c0).astype(np.float64)
    v = p - d[0]
    t = v @ d[3] / (d[3] @ d[3])
    ux = (v @ d[1]) / (t * (d[1] @ d[1]))
    uy = (v @ d[2]) / (t * (d[2] @ d[2]))
    xc, yc = (ux + 1) * 0.5 * W, (uy + 1) * 0.5 * H
    inside = ok & (t > 0) & (xc >= 0) & (xc < W) & (yc >= 0) & (yc < H)
    want = np.where(inside, np.floor(xc).astype(np.int64) | (np.floor(yc).astype(np.int64) << 16), 0xFFFFFFFF)
    near_edge = (np.abs(xc - np.round(xc)) < 1e-3) | (np.abs(yc - np.round(yc)) < 1e-3)
    assert ok.mean() > 0.5
    assert (pxy[ok & ~near_edge] == want[ok & ~near_edge]).all()
    assert (pxy[~ok] == 0xFFFFFFFF).all()
    moved = inside & (pxy != (np.arange(W * H) % W) | ((np.arange(W * H) // W) << 16))
    assert moved.mean() > 0.5  # the camera moved: most pixels come from elsewhere


def test_oracle_rejects_unknown_motion_mode():
    desc, cam = scenes.cornell_box()
    with pytest.raises(RuntimeError):
        op.Oracle.from_scene(desc, W, H, small_config_params(scene_size_of(desc), motion_mode=3))


# ---- GPU parity -----------------------------------------------------------------

def _random_motion(seed):
    rng = np.random.default_rng(seed)
    mv = rng.normal(0.0, 3.0, (H, W, 2)).astype(np.float32)
    mv[rng.random((H, W)) < 0.02] = np.nan
    mv[rng.random((H, W)) < 0.02] = 1e9
    return mv


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [_abi.STORAGE_FP32, _abi.STORAGE_FP16])
@pytest.mark.parametrize("mode", [_abi.MOTION_VECTORS, _abi.MOTION_REPROJECT])
def test_motion_parity(cuda_device, mode, storage):
    from test_parity_gpu import run_parity

    desc, cam = scenes.cornell_box()
    p = small_config_params(scene_size_of(desc), motion_mode=mode, storage=storage)
    motion = _random_motion(7) if mode == _abi.MOTION_VECTORS else None
    run_parity(desc, cam, p, W, H, 4, lambda c, f: orbit(c, f, 30), motion=motion,
               graph=lambda f: f % 2 == 0)


@pytest.mark.gpu
def test_motion_parity_large_config(cuda_device):
    from helpers import large_config_params, small_sphere_room
    from test_parity_gpu import run_parity

    desc, cam = small_sphere_room()
    p = large_config_params(scene_size_of(desc), gather_radius=0.3, motion_mode=_abi.MOTION_REPROJECT)
    run_parity(desc, cam, p, 64, 48, 4, lambda c, f: orbit(c, f, 120))


@pytest.mark.gpu
def test_motion_vectors_required(cuda_device):
    import torch

    from crisoptix_b200 import CrisbError, Renderer, Scene

    desc, cam = scenes.cornell_box()
    r = Renderer(W, H, Scene(desc), small_config_params(scene_size_of(desc), motion_mode=_abi.MOTION_VECTORS))
    out = torch.zeros(W * H * 3, device="cuda")
    with pytest.raises(CrisbError):
        r.launch_frame(cam, out.data_ptr())
