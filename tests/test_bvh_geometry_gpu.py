"""Hits of the device-built trees against testing every triangle, on
geometry that stresses the trees rather than the renderer: a flat
axis-aligned grid (zero extent on one axis, so the compressed nodes' grid
step comes from the box margin alone), mixed scales (a large quad beside
clusters of triangles a million times smaller, far from the origin, where a
grid step is close to the float spacing of the coordinates), stacks of
identical triangles (ties go to the lower triangle index), fans of many
triangles around one vertex, a single triangle, and a random soup.  Both
device formats: compressed 8-wide nodes (the default) and 4-wide nodes."""
import numpy as np
import pytest

import oracle_py as op
from crisoptix_b200 import Scene, _abi, scenes
from helpers import first_mismatch, make_params, random_rays, surface_rays

pytestmark = pytest.mark.gpu


def soup(P: np.ndarray, name: str) -> scenes.Scene:
    """Scene of the (T, 9) triangle positions, one diffuse material, the
    first triangle an emitter."""
    P = np.asarray(P, np.float32).reshape(-1, 3, 3)
    n = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    n = np.where(ln > 0, n / np.maximum(ln, 1e-30), np.array([[0.0, 1.0, 0.0]]))
    N = np.repeat(n[:, None, :], 3, axis=1).astype(np.float32)
    T = len(P)
    idx = np.arange(3 * T, dtype=np.uint32).reshape(T, 3)
    mats = np.stack([scenes._material((0.6, 0.6, 0.6), emission=(1.0, 1.0, 1.0))])
    return scenes.Scene(P.reshape(-1, 3), N.reshape(-1, 3), idx, np.zeros(T, np.uint32), mats,
                        np.zeros((0, 2), np.uint32), [], [((1.0, 1.0, 1.0), 0, 1)],
                        P[:1].reshape(1, 9).astype(np.float32), name=name)


def flat_grid():
    """40 x 40 quads in the plane y = 0 (3,200 triangles)."""
    tris = []
    for i in range(40):
        for j in range(40):
            x0, z0, x1, z1 = i * 0.05 - 1.0, j * 0.05 - 1.0, (i + 1) * 0.05 - 1.0, (j + 1) * 0.05 - 1.0
            tris.append([x0, 0, z0, x1, 0, z0, x1, 0, z1])
            tris.append([x0, 0, z0, x1, 0, z1, x0, 0, z1])
    return np.asarray(tris, np.float32)


def mixed_scales():
    """A 2000-unit floor quad and 50 clusters of 20 triangles of size 1e-3
    around points 300-700 units from the origin."""
    rng = np.random.default_rng(7)
    tris = [[-1000, -1, -1000, 1000, -1, -1000, 1000, -1, 1000], [-1000, -1, -1000, 1000, -1, 1000, -1000, -1, 1000]]
    for _ in range(50):
        c = rng.uniform(-1, 1, 3)
        c = c / np.linalg.norm(c) * rng.uniform(300, 700)
        for _ in range(20):
            base = c + rng.normal(size=3) * 5e-3
            tris.append(np.concatenate([base, base + rng.normal(size=3) * 1e-3, base + rng.normal(size=3) * 1e-3]))
    return np.asarray(tris, np.float32)


def stacks_and_fans():
    """Ten copies of each of 30 triangles (ties), and 6 fans of 200 thin
    triangles around one vertex each."""
    rng = np.random.default_rng(8)
    tris = []
    for _ in range(30):
        t = rng.uniform(-1, 1, 9)
        tris += [t] * 10
    for _ in range(6):
        c = rng.uniform(-1, 1, 3)
        for k in range(200):
            a0, a1 = 2 * np.pi * k / 200, 2 * np.pi * (k + 1) / 200
            tris.append(np.concatenate([c, c + 0.3 * np.array([np.cos(a0), 0.1, np.sin(a0)]),
                                        c + 0.3 * np.array([np.cos(a1), 0.1, np.sin(a1)])]))
    return np.asarray(tris, np.float32)


def single():
    return np.asarray([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32)


def random_soup():
    rng = np.random.default_rng(9)
    c = rng.uniform(-4, 4, (5000, 1, 3))
    s = np.exp(rng.uniform(np.log(1e-3), np.log(1.0), (5000, 1, 1)))
    return (c + rng.normal(size=(5000, 3, 3)) * s).reshape(-1, 9).astype(np.float32)


GEOMETRY = {"flat_grid": flat_grid, "mixed_scales": mixed_scales, "stacks_and_fans": stacks_and_fans,
            "single": single, "random_soup": random_soup}


def grazing_rays(n: int, seed: int) -> np.ndarray:
    """Rays starting on or just above the plane y = 0, directions in the
    plane or a hair off it, and axis-aligned ones."""
    rng = np.random.default_rng(seed)
    o = np.zeros((n, 3), np.float32)
    o[:, 0] = rng.uniform(-1.2, 1.2, n)
    o[:, 2] = rng.uniform(-1.2, 1.2, n)
    o[:, 1] = rng.choice([0.0, 1e-6, -1e-6, 1e-3], n)
    d = rng.normal(size=(n, 3))
    d[:, 1] = rng.choice([0.0, 1e-7, -1e-7, -1e-3, -0.5], n)
    d[: n // 8] = np.eye(3)[rng.integers(0, 3, n // 8)] * rng.choice([-1, 1], (n // 8, 1))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 1e-4
    rays[:, 4:7] = d
    rays[:, 7] = 1e16
    return rays


def aimed_rays(desc, n: int, seed: int) -> np.ndarray:
    """Rays from points around the scene's bounding box (grown by half its
    diagonal) toward random points of random triangles."""
    rng = np.random.default_rng(seed)
    pos, _, _ = desc.flatten()
    tri = pos.reshape(-1, 3, 3)
    lo, hi = tri.reshape(-1, 3).min(0), tri.reshape(-1, 3).max(0)
    g = 0.5 * np.linalg.norm(hi - lo) + 1e-3
    o = rng.uniform(lo - g, hi + g, (n, 3))
    t = rng.integers(0, len(tri), n)
    w = rng.random((n, 3))
    w /= w.sum(1, keepdims=True)
    p = (w[:, :, None] * tri[t]).sum(1)
    d = p - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 1e-3
    rays[:, 4:7] = d
    rays[:, 7] = 1e16
    return rays


def gpu_trace(scene, rays, any_hit):
    from test_parity_gpu import gpu_trace as trace
    return trace(scene, rays, any_hit)


@pytest.mark.parametrize("builder", [_abi.BVH_DEVICE, _abi.BVH_DEVICE_WIDE4])
@pytest.mark.parametrize("which", list(GEOMETRY))
def test_tree_hits_equal_brute_force(cuda_device, which, builder):
    desc = soup(GEOMETRY[which](), which)
    sc = Scene(desc, builder=builder)
    info = sc.bvh_info()
    assert info["format"] == (_abi.BVH_FORMAT_COMPRESSED8 if builder == _abi.BVH_DEVICE else _abi.BVH_FORMAT_WIDE4)
    o = op.Oracle.from_scene(desc, 4, 4, make_params(sc.scene_size), triangles=sc.read_triangles())
    sets = [random_rays(desc, 1 << 15, seed=31), aimed_rays(desc, 1 << 15, seed=34)]
    if which == "flat_grid":
        sets.append(grazing_rays(1 << 15, seed=32))
    if len(desc.indices) > 1:
        sets.append(surface_rays(desc, 1 << 15, seed=33))
    hit_any = 0
    for rays in sets:
        for any_hit in (False, True):
            g = gpu_trace(sc, rays, any_hit)
            c = o.trace(rays, any_hit=any_hit, brute=True)
            mm = first_mismatch(g, c)
            assert mm is None, (which, any_hit, mm)
            hit_any += int((g["prim"] != _abi.INVALID_PRIM).sum())
    assert hit_any > 0
