"""GPU parity at the workloads' stated sizes, not reduced ones.

Small: the procedural Cornell box at 256x256 for 16 frames, seed 0 (max depth
4, prefix length 1, 1 temporal + 1 spatial pass of 3 neighbours in a 30 px
window).  Large: the 1,310,988-triangle sphere room at 1920x1080 over the
first three frames of the 60-frame orbit, seed 1 (max depth 8, prefix length
2, k = 8, 1 temporal + 2 spatial passes of 5 neighbours), in FP32 and in FP16
reservoir storage.  Every state buffer and the image must equal the oracle's
bit for bit after every frame -- the scale-dependent parts (queue capacities,
32-bit index products, the endpoint structure over 2 M entries, a
383 K-node scene tree) are exercised at the size the benchmark runs.
"""
import pytest

from crisoptix_b200 import Scene, _abi, scenes
from helpers import large_config_params, orbit, scene_size_of, small_config_params, static
from test_parity_gpu import run_parity

pytestmark = pytest.mark.gpu


def test_small_config_at_stated_size(cuda_device):
    desc, cam = scenes.cornell_box()
    p = small_config_params(scene_size_of(desc))
    out = run_parity(desc, cam, p, 256, 256, 16, static)
    assert out.mean() > 0.5


@pytest.mark.parametrize("storage", [_abi.STORAGE_FP32, _abi.STORAGE_FP16])
def test_large_config_at_stated_size(cuda_device, storage):
    desc, cam = scenes.sphere_room(num_spheres=64, subdiv=5, num_emitters=256, seed=1)
    assert Scene(desc).num_triangles == 1310988
    p = large_config_params(scene_size_of(desc), storage=storage)
    out = run_parity(desc, cam, p, 1920, 1080, 3, lambda c, f: orbit(c, f, 60))
    assert out.mean() > 0.0
