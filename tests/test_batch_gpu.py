"""Batched views: one CUDA graph with a branch per view gives every view the
same state and image as rendering it alone."""
import numpy as np
import pytest
import torch

from crisoptix_b200 import Batch, Renderer, Scene, _abi, scenes
from helpers import large_config_params, orbit, scene_size_of, small_sphere_room

STATE_BUFS = [_abi.BUF_PREFIX_RES_FRONT, _abi.BUF_PREFIX_RES_BACK, _abi.BUF_SUFFIX_RES_FRONT, _abi.BUF_GBUFFER,
              _abi.BUF_NEIGHBORS, _abi.BUF_NEIGHBOR_COUNT]


@pytest.mark.gpu
def test_batch_matches_single_views(cuda_device):
    desc, cam = small_sphere_room()
    sc = Scene(desc)
    size = scene_size_of(desc)
    views = [(48, 40, large_config_params(size, gather_radius=0.3)),
             (32, 32, large_config_params(size, gather_radius=0.3, storage=_abi.STORAGE_FP16)),
             (40, 24, large_config_params(size, gather_radius=0.2, suffix_spatial_rounds=1, gather_m=4))]
    batched = [Renderer(w, h, sc, p) for w, h, p in views]
    single = [Renderer(w, h, sc, p) for w, h, p in views]
    batch = Batch(batched)
    outs_b = [torch.zeros(w * h * 3, dtype=torch.float32, device="cuda") for w, h, _ in views]
    outs_s = [torch.zeros(w * h * 3, dtype=torch.float32, device="cuda") for w, h, _ in views]
    for f in range(3):
        cams = [orbit(cam, f + 7 * k, 120) for k in range(len(views))]
        batch.render(cams, [o.data_ptr() for o in outs_b])
        for r, c, o in zip(single, cams, outs_s):
            r.launch_frame(c, o.data_ptr())
        torch.cuda.synchronize()
        for k in range(len(views)):
            batched[k].check_device_errors()
            assert outs_b[k].cpu().numpy().tobytes() == outs_s[k].cpu().numpy().tobytes(), (f, k)
            for b in STATE_BUFS:
                assert batched[k].debug_read(b).tobytes() == single[k].debug_read(b).tobytes(), (f, k, b)


@pytest.mark.gpu
def test_batch_rejects_bad_input(cuda_device):
    desc, cam = scenes.cornell_box()
    sc = Scene(desc)
    r = Renderer(16, 16, sc, large_config_params(scene_size_of(desc)))
    with pytest.raises(Exception):
        Batch([r, r])
    b = Batch([r])
    with pytest.raises(Exception):
        b.render([cam], [0])


@pytest.mark.gpu
def test_batch_with_srgb_output_and_reprojection(cuda_device):
    """Batched views with the sRGB epilogue and temporal reprojection on: each
    view's bytes and state equal the same view rendered alone."""
    desc, cam = small_sphere_room()
    sc = Scene(desc)
    size = scene_size_of(desc)
    views = [(48, 40, large_config_params(size, gather_radius=0.3, motion_mode=_abi.MOTION_REPROJECT)),
             (33, 17, large_config_params(size, gather_radius=0.3))]
    batched = [Renderer(w, h, sc, p) for w, h, p in views]
    single = [Renderer(w, h, sc, p) for w, h, p in views]
    batch = Batch(batched)
    hdr_b = [torch.zeros(w * h * 3, dtype=torch.float32, device="cuda") for w, h, _ in views]
    hdr_s = [torch.zeros(w * h * 3, dtype=torch.float32, device="cuda") for w, h, _ in views]
    srgb_b = [torch.zeros(w * h * 3, dtype=torch.uint8, device="cuda") for w, h, _ in views]
    srgb_s = [torch.zeros(w * h * 3, dtype=torch.uint8, device="cuda") for w, h, _ in views]
    for r, o in zip(batched, srgb_b):
        r.set_srgb_output(o.data_ptr())
    for r, o in zip(single, srgb_s):
        r.set_srgb_output(o.data_ptr())
    for f in range(3):
        cams = [orbit(cam, f + 11 * k, 120) for k in range(len(views))]
        batch.render(cams, [o.data_ptr() for o in hdr_b])
        for r, c, o in zip(single, cams, hdr_s):
            r.launch_frame(c, o.data_ptr())
        torch.cuda.synchronize()
        for k in range(len(views)):
            assert hdr_b[k].cpu().numpy().tobytes() == hdr_s[k].cpu().numpy().tobytes(), (f, k)
            assert (srgb_b[k].cpu() == srgb_s[k].cpu()).all(), (f, k)
            assert int(srgb_b[k].sum()) > 0
            for b in STATE_BUFS:
                assert batched[k].debug_read(b).tobytes() == single[k].debug_read(b).tobytes(), (f, k, b)
