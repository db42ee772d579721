"""Launch-shape tuning: traversal grid, traversal block size and job capacity
change no result, and autotuning leaves the renderer's own frame sequence
untouched."""
import numpy as np
import pytest
import torch

from crisoptix_b200 import Renderer, Scene, _abi
from helpers import large_config_params, orbit, scene_size_of, small_sphere_room

BUFS = [_abi.BUF_PREFIX_RES_FRONT, _abi.BUF_SUFFIX_RES_FRONT, _abi.BUF_GBUFFER]


@pytest.mark.gpu
def test_trace_grid_and_autotune_do_not_change_results(cuda_device):
    desc, cam = small_sphere_room()
    sc = Scene(desc)
    p = large_config_params(scene_size_of(desc), gather_radius=0.3)
    ref = Renderer(48, 40, sc, p)
    ref.set_trace_grid(1)
    tuned = Renderer(48, 40, sc, p)
    out_r = torch.zeros(48 * 40 * 3, device="cuda")
    out_t = torch.zeros(48 * 40 * 3, device="cuda")
    for f in range(4):
        c = orbit(cam, f, 120)
        if f == 1:
            chosen = tuned.autotune(c, frames=1)
            assert chosen["trace_grid"] in (1, 2, 4, 8, 16)
            assert chosen["trace_block"] in (64, 128, 256)
            assert 1 <= chosen["jobs_per_pixel"] <= 16 and chosen["frame_ms"] > 0
            assert tuned.job_capacity() == chosen["jobs_per_pixel"]
        ref.launch_frame(c, out_r.data_ptr())
        tuned.launch_frame(c, out_t.data_ptr())
        torch.cuda.synchronize()
        assert out_r.cpu().numpy().tobytes() == out_t.cpu().numpy().tobytes(), f
        for b in BUFS:
            assert ref.debug_read(b).tobytes() == tuned.debug_read(b).tobytes(), (f, b)


@pytest.mark.gpu
@pytest.mark.parametrize("threads", [64, 256])
def test_trace_block_sizes_do_not_change_results(cuda_device, threads):
    desc, cam = small_sphere_room()
    sc = Scene(desc)
    p = large_config_params(scene_size_of(desc), gather_radius=0.3)
    a, b = Renderer(48, 40, sc, p), Renderer(48, 40, sc, p)
    b.set_trace_block(threads)
    oa, ob = torch.zeros(48 * 40 * 3, device="cuda"), torch.zeros(48 * 40 * 3, device="cuda")
    for f in range(3):
        c = orbit(cam, f, 120)
        a.launch_frame(c, oa.data_ptr())
        b.launch_frame(c, ob.data_ptr())
        torch.cuda.synchronize()
        assert oa.cpu().numpy().tobytes() == ob.cpu().numpy().tobytes(), f


@pytest.mark.gpu
def test_spatial_count_autotuner_fits_the_budget(cuda_device):
    """crisb_autotune_spatial: a budget every candidate fits picks the largest
    count (16), one none fits picks the cheapest (1); the choice is set on
    the renderer, which keeps rendering with it, and its frame time is
    within the budget it was picked for."""
    desc, cam = small_sphere_room()
    sc = Scene(desc)
    p = large_config_params(scene_size_of(desc), max_path_len=4)
    r = Renderer(96, 64, sc, p)
    out = torch.zeros(96 * 64 * 3, device="cuda")
    r.launch_frame(cam, out.data_ptr())
    big = r.autotune_spatial(cam, budget_ms=1e6, frames=2)
    assert big["count"] == 16 and r.params.suffix_spatial_count == 16, big
    assert 0.0 < big["frame_ms"] < 1e6
    r.launch_frame(cam, out.data_ptr())
    tiny = r.autotune_spatial(cam, budget_ms=1e-4, frames=2)
    assert tiny["count"] == 1 and r.params.suffix_spatial_count == 1, tiny
    r.launch_frame(cam, out.data_ptr())
    budget = 0.5 * (big["frame_ms"] + tiny["frame_ms"])
    mid = r.autotune_spatial(cam, budget_ms=budget, frames=2)
    # within the budget, or the cheapest when timing noise puts every count over it
    assert 1 <= mid["count"] <= 16 and (mid["count"] == 1 or mid["frame_ms"] <= budget), mid
    r.launch_frame(cam, out.data_ptr())
    r.check_device_errors()
    torch.cuda.synchronize()
    assert np.isfinite(out.cpu().numpy()).all()
    with pytest.raises(RuntimeError):
        Renderer(32, 24, sc, large_config_params(scene_size_of(desc), suffix_enable_spatial=0)).autotune_spatial(
            cam, budget_ms=10.0)
