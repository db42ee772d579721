"""Shared helpers for the parity tests: workloads and record comparison."""
from __future__ import annotations

import math

import numpy as np

from crisoptix_b200 import _abi, scenes


def make_params(scene_size: float, **kw) -> _abi.Params:
    """Reference defaults (src/Renderer.cpp:34-58) without touching the CUDA
    library, then overrides."""
    p = _abi.Params()
    p.renderer_type = _abi.PATH_TRACER
    p.nee_prob = 0.3
    p.max_path_len = 8
    p.enable_accum = 0
    p.recon_min_distance = 0.01 * scene_size
    p.recon_min_roughness = 0.2
    p.prefix_len = 2
    p.prefix_enable_temporal = 1
    p.prefix_enable_spatial = 0
    p.prefix_spatial_count = 1
    p.prefix_spatial_rounds = 1
    p.suffix_enable_temporal = 1
    p.suffix_enable_spatial = 1
    p.suffix_spatial_count = 1
    p.suffix_spatial_rounds = 1
    p.gather_n = 1
    p.gather_m = 1
    p.gather_radius = 0.01
    p.gather_radius_type = _abi.RADIUS_PATH_LENGTH
    p.window_radius = 10
    p.storage = _abi.STORAGE_FP32
    p.seed = 0
    for k, v in kw.items():
        assert hasattr(p, k), k
        setattr(p, k, v)
    return p


def small_config_params(scene_size: float, **kw) -> _abi.Params:
    """Small (Cornell) workload: max depth 4, prefix length 1, 1 temporal +
    1 spatial pass with 3 neighbours in a 30 px window, seed 0."""
    base = dict(renderer_type=_abi.CONDITIONAL_RESTIR, max_path_len=4, prefix_len=1, suffix_spatial_count=3,
                suffix_spatial_rounds=1, window_radius=30, seed=0)
    base.update(kw)
    return make_params(scene_size, **base)


def large_config_params(scene_size: float, **kw) -> _abi.Params:
    """Large workload: max depth 8, prefix kNN k = 8, 1 temporal + 2 spatial
    passes of 5 neighbours, seed 1."""
    base = dict(renderer_type=_abi.CONDITIONAL_RESTIR, max_path_len=8, prefix_len=2, gather_m=9,
                suffix_spatial_count=5, suffix_spatial_rounds=2, seed=1)
    base.update(kw)
    return make_params(scene_size, **base)


def small_sphere_room(seed: int = 5):
    """A reduced version of the large scene for parity runs."""
    return scenes.sphere_room(num_spheres=8, subdiv=2, num_emitters=16, seed=seed, room=(6.0, 3.0, 6.0),
                              aspect=1.0)


def scene_size_of(desc) -> float:
    pos, _, _ = desc.flatten()
    p = pos.reshape(-1, 3)
    lo = np.minimum(p.min(axis=0), 0.0)
    hi = np.maximum(p.max(axis=0), 0.0)
    return float(np.linalg.norm(hi - lo))


def random_rays(desc, n: int, seed: int, origin_box=None) -> np.ndarray:
    rng = np.random.default_rng(seed)
    pos, _, _ = desc.flatten()
    p = pos.reshape(-1, 3)
    lo, hi = p.min(axis=0), p.max(axis=0)
    if origin_box is not None:
        lo, hi = np.asarray(origin_box[0]), np.asarray(origin_box[1])
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # a few axis-aligned and grazing directions
    d[: n // 16] = np.eye(3)[rng.integers(0, 3, n // 16)] * rng.choice([-1, 1], (n // 16, 1))
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 1e-3
    rays[:, 4:7] = d
    rays[:, 7] = 1e16
    return rays


def first_mismatch(a: np.ndarray, b: np.ndarray):
    """Index and field name of the first bytewise difference of two record
    arrays, or None."""
    assert a.dtype == b.dtype and a.shape == b.shape
    if a.size == 0:
        return None
    ab = a.view(np.uint8).reshape(len(a), -1)
    bb = b.view(np.uint8).reshape(len(b), -1)
    bad = np.nonzero((ab != bb).any(axis=1))[0]
    if len(bad) == 0:
        return None
    i = int(bad[0])
    fields = []

    def walk(dt, off, prefix):
        if dt.fields is None:
            n = dt.itemsize
            if (ab[i, off:off + n] != bb[i, off:off + n]).any():
                fields.append(prefix)
            return
        for name, (sub, o) in dt.fields.items():
            walk(sub, off + o, prefix + "." + name if prefix else name)

    walk(a.dtype, 0, "")
    return i, fields, len(bad)


def orbit(cam, frame, frames_per_orbit=60):
    return scenes.orbit_camera(cam, frame, frames_per_orbit)


def static(cam, frame):
    return scenes.Camera(cam.pos, cam.view_dir, cam.up, cam.aspect, cam.fov, False)


TWO_PI = 2.0 * math.pi


def surface_rays(desc, n: int, seed: int) -> np.ndarray:
    """Rays between points on the scene's triangles, as shadow and
    reconnection rays run them: from a surface point (tmin 1e-3) to another
    surface point at tmax = their distance.  A sixth of the endpoints sit on a
    triangle edge and a sixth on a vertex, so on axis-aligned geometry many
    rays lie in a face plane (a zero direction component) and end on an edge:
    the configurations where a box test can disagree with the triangle test."""
    rng = np.random.default_rng(seed)
    pos, _, _ = desc.flatten()
    tri = pos.reshape(-1, 3, 3).astype(np.float32)

    def points(m):
        t = rng.integers(0, len(tri), m)
        r = rng.random((m, 3)).astype(np.float32)
        k = rng.integers(0, 6, m)
        r[k == 0, 0] = 0.0
        r[k == 1] = [1.0, 0.0, 0.0]
        r /= r.sum(1, keepdims=True)
        return (r[:, 0:1] * tri[t, 0] + r[:, 1:2] * tri[t, 1] + r[:, 2:3] * tri[t, 2]).astype(np.float32)

    a, b = points(n), points(n)
    d = (b - a).astype(np.float32)
    ln = np.sqrt((d * d).sum(1)).astype(np.float32)
    keep = ln > 1e-3
    a, d, ln = a[keep], d[keep], ln[keep]
    d = (d / ln[:, None]).astype(np.float32)
    rays = np.zeros((len(a), 8), np.float32)
    rays[:, 0:3] = a
    rays[:, 3] = 1e-3
    rays[:, 4:7] = d
    rays[:, 7] = ln
    return rays
