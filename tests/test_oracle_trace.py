"""The oracle's BVH traversal against brute force over every triangle (CPU)."""
import numpy as np
import pytest

import oracle_py as op
from crisoptix_b200 import scenes
from helpers import make_params, random_rays, scene_size_of, small_sphere_room


@pytest.mark.parametrize("which", ["cornell", "spheres"])
def test_bvh_closest_and_occlusion_match_bruteforce(which):
    desc = scenes.cornell_box()[0] if which == "cornell" else small_sphere_room()[0]
    o = op.Oracle.from_scene(desc, 4, 4, make_params(scene_size_of(desc)))
    rays = random_rays(desc, 4096, seed=11)
    a, b = o.trace(rays), o.trace(rays, brute=True)
    assert (a["prim"] != 0xFFFFFFFF).mean() > 0.5
    assert a.tobytes() == b.tobytes()
    short = rays.copy()
    short[:, 7] = np.random.default_rng(2).uniform(0.01, 2.0, len(rays))
    assert o.trace(short, any_hit=True).tobytes() == o.trace(short, any_hit=True, brute=True).tobytes()


def test_watertight_shared_edge():
    # rays through the shared diagonal of a quad must hit one of its triangles
    desc, _ = scenes.cornell_box()
    o = op.Oracle.from_scene(desc, 4, 4, make_params(scene_size_of(desc)))
    t = np.linspace(-0.49, 0.49, 257, dtype=np.float32)
    rays = np.zeros((len(t), 8), np.float32)
    rays[:, 0] = t
    rays[:, 1] = 0.5
    rays[:, 2] = -t  # floor diagonal from (-0.5,0,0.5) to (0.5,0,-0.5)
    rays[:, 3] = 1e-3
    rays[:, 5] = -1.0
    rays[:, 7] = 1e16
    h = o.trace(rays)
    assert (h["prim"] != 0xFFFFFFFF).all()  # nothing slips through the diagonal
    off_box = (t < 0.0) | (t > 0.34)  # the short box stands on part of the diagonal
    assert set(int(p) for p in h["prim"][off_box]) <= {0, 1}
