"""GPU parity: the CUDA frame loop against the oracle, through the C ABI.

Discrete state (hit triangle ids, reconnection indices, flags, reservoir
selections, neighbour lists, RNG states) must match bit for bit; so do all
floating-point record fields and the image, because both sides evaluate the
same IEEE operations in the same order.  The image check also states the
value tolerance the frame loop promises (1e-4 relative).
"""
import numpy as np
import pytest
import torch

import oracle_py as op
from crisoptix_b200 import Renderer, Scene, _abi, scenes
from helpers import first_mismatch, large_config_params, make_params, orbit, random_rays, scene_size_of, \
    small_config_params, small_sphere_room, static

pytestmark = pytest.mark.gpu

STATE_BUFS = [_abi.BUF_PREFIX_RES_FRONT, _abi.BUF_PREFIX_RES_BACK, _abi.BUF_CANON_PREFIX, _abi.BUF_SUFFIX_RES_FRONT,
              _abi.BUF_CANON_SUFFIX, _abi.BUF_GBUFFER, _abi.BUF_NEIGHBORS, _abi.BUF_NEIGHBOR_COUNT]
RTOL = 1e-4


def gpu_trace(scene: Scene, rays: np.ndarray, any_hit: bool) -> np.ndarray:
    r = torch.from_numpy(np.ascontiguousarray(rays, np.float32)).cuda()
    h = torch.zeros((len(rays), 4), dtype=torch.int32, device="cuda")
    scene.trace(r.data_ptr(), h.data_ptr(), len(rays), any_hit)
    torch.cuda.synchronize()
    return h.cpu().numpy().view(_abi.TRACE_HIT_DTYPE).reshape(-1)


BUILDERS = [_abi.BVH_DEVICE, _abi.BVH_DEVICE_WIDE4]


def make_scene(desc, builder):
    """Scene built by `builder`; the default build of these scenes must give
    compressed nodes, the others 4-wide ones."""
    sc = Scene(desc, builder=builder)
    info = sc.bvh_info()
    if builder == _abi.BVH_DEVICE:
        assert info["format"] == _abi.BVH_FORMAT_COMPRESSED8 and info["node_bytes"] == 80, info
    else:
        assert info["format"] == _abi.BVH_FORMAT_WIDE4 and info["node_bytes"] == 128, info
    return sc


@pytest.mark.parametrize("builder", BUILDERS)
@pytest.mark.parametrize("which", ["cornell", "spheres"])
def test_traversal_hits_bit_exact(cuda_device, which, builder):
    desc = scenes.cornell_box()[0] if which == "cornell" else small_sphere_room()[0]
    sc = make_scene(desc, builder)
    tri = sc.read_triangles()
    o = op.Oracle.from_scene(desc, 4, 4, make_params(sc.scene_size), triangles=tri)
    rays = random_rays(desc, 1 << 15, seed=3)
    g, c = gpu_trace(sc, rays, False), o.trace(rays)
    assert (g["prim"] != _abi.INVALID_PRIM).mean() > 0.5
    assert first_mismatch(g, c) is None, first_mismatch(g, c)
    rays[:, 7] = np.random.default_rng(4).uniform(0.01, 3.0, len(rays))
    assert gpu_trace(sc, rays, True).tobytes() == o.trace(rays, any_hit=True).tobytes()


def test_flattened_instances_match_float64_reference(cuda_device):
    desc, _ = small_sphere_room()
    pos, nrm, mat = Scene(desc).read_triangles()
    rp, rn, rm = desc.flatten()
    np.testing.assert_allclose(pos, rp, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(nrm, rn, rtol=1e-5, atol=1e-5)
    assert (mat == rm).all()


def run_parity(desc, cam, params, W, H, frames, cam_fn, change_params=None, timing=0, graph=lambda f: True,
               motion=None, jobs_per_pixel=None, builder=_abi.BVH_DEVICE):
    sc = make_scene(desc, builder)
    tri = sc.read_triangles()
    o = op.Oracle.from_scene(desc, W, H, params, triangles=tri)
    r = Renderer(W, H, sc, params)
    if jobs_per_pixel is not None:
        r.set_job_capacity(jobs_per_pixel)
        assert r.job_capacity() == jobs_per_pixel
    r.set_timing(timing)
    if motion is not None:  # (H, W, 2) motion vectors for MOTION_VECTORS
        mv_d = torch.from_numpy(np.ascontiguousarray(motion, np.float32)).cuda()
        r.set_motion_vectors(mv_d.data_ptr())
        o.set_motion_vectors(motion)
    out_d = torch.zeros(H * W * 3, dtype=torch.float32, device="cuda")
    out_h = np.zeros((H, W, 3), np.float32)
    for f in range(frames):
        if change_params and f in change_params:
            params = change_params[f]
            r.params = params
            o.set_params(params)
        c = cam_fn(cam, f)
        r.set_graph(graph(f))
        r.launch_frame(c, out_d.data_ptr())
        torch.cuda.synchronize()
        o.render_frame(c, out_h)
        r.check_device_errors()
        assert r.get_frame_idx() == o.frame_index() and r.frame_random() == o.frame_random()
        for b in STATE_BUFS:
            g, c2 = r.debug_read(b), o.dump(b)
            mm = first_mismatch(g, c2)
            assert mm is None, f"frame {f} buffer {b}: first mismatch at {mm}"
        img = out_d.cpu().numpy().reshape(H, W, 3)
        np.testing.assert_allclose(img, out_h, rtol=RTOL, atol=1e-6)
        assert img.tobytes() == out_h.tobytes()
        if timing:
            st = r.stats()
            assert st["total_ms"] > 0 and st["trace_ms"] > 0
            if timing >= 2:
                assert st["closest_rays"] >= W * H // 2 and st["shadow_rays"] > 0
    return out_h


def test_small_config_cornell_conditional_restir(cuda_device):
    desc, cam = scenes.cornell_box()
    p = small_config_params(scene_size_of(desc))
    out = run_parity(desc, cam, p, 64, 64, 4, static)
    assert out.mean() > 0.5


def test_cornell_with_endpoint_search(cuda_device):
    desc, cam = scenes.cornell_box()
    p = small_config_params(scene_size_of(desc), gather_m=9, gather_radius=0.5, gather_n=2)
    run_parity(desc, cam, p, 48, 40, 3, static)


def test_large_config_reduced_scene_orbit(cuda_device):
    desc, cam = small_sphere_room()
    p = large_config_params(scene_size_of(desc), gather_radius=0.3)
    run_parity(desc, cam, p, 64, 48, 4, lambda c, f: orbit(c, f, 120))


@pytest.mark.parametrize("rtype", [_abi.PATH_TRACER, _abi.RESTIR_PT])
def test_other_renderer_types(cuda_device, rtype):
    desc, cam = scenes.cornell_box()
    p = make_params(scene_size_of(desc), renderer_type=rtype, max_path_len=5, prefix_enable_spatial=1,
                    prefix_spatial_count=3, prefix_spatial_rounds=2, enable_accum=1)
    run_parity(desc, cam, p, 40, 40, 3, static)


def test_param_change_between_frames(cuda_device):
    desc, cam = scenes.cornell_box()
    p0 = small_config_params(scene_size_of(desc))
    p1 = small_config_params(scene_size_of(desc), gather_m=4, gather_radius=0.4, suffix_spatial_rounds=2,
                             prefix_enable_spatial=1, prefix_spatial_count=2)
    run_parity(desc, cam, p0, 32, 32, 4, static, change_params={2: p1})


def test_timing_and_ray_counters_do_not_change_results(cuda_device):
    desc, cam = small_sphere_room()
    p = large_config_params(scene_size_of(desc), gather_radius=0.3)
    run_parity(desc, cam, p, 48, 40, 3, lambda c, f: orbit(c, f, 120), timing=2)


def test_direct_launches_match(cuda_device):
    """Frames launched kernel by kernel instead of as one CUDA graph."""
    desc, cam = small_sphere_room()
    p = large_config_params(scene_size_of(desc), gather_radius=0.3)
    run_parity(desc, cam, p, 48, 40, 3, lambda c, f: orbit(c, f, 120), graph=lambda f: False)


def test_graph_and_direct_frames_interleaved(cuda_device):
    """Graph frames, direct frames and a parameter change that alters the
    graph's shape, in one sequence."""
    desc, cam = scenes.cornell_box()
    p0 = small_config_params(scene_size_of(desc))
    p1 = small_config_params(scene_size_of(desc), gather_m=4, gather_radius=0.4, suffix_spatial_rounds=2)
    run_parity(desc, cam, p0, 32, 32, 6, static, change_params={3: p1}, graph=lambda f: f % 3 != 1)


@pytest.mark.parametrize("jobs_per_pixel", [0, 1])
def test_shift_jobs_beyond_capacity_give_the_same_results(cuda_device, jobs_per_pixel):
    """With no machine capacity every shift job runs in the overflow kernel,
    with one job per pixel most passes overflow part of their list: the
    frames must not change."""
    desc, cam = small_sphere_room()
    p = large_config_params(scene_size_of(desc), gather_radius=0.3)
    run_parity(desc, cam, p, 48, 40, 3, lambda c, f: orbit(c, f, 120), jobs_per_pixel=jobs_per_pixel)


@pytest.mark.parametrize("builder", [_abi.BVH_HOST, _abi.BVH_DEVICE_WIDE4])
def test_other_trees_give_the_same_frames(cuda_device, builder):
    desc, cam = small_sphere_room()
    p = large_config_params(scene_size_of(desc), gather_radius=0.3)
    run_parity(desc, cam, p, 48, 40, 2, lambda c, f: orbit(c, f, 120), builder=builder)


def test_compressed_tree_layout(cuda_device):
    """The compressed build makes 80-byte nodes, fewer of them than the
    4-wide build of the same scene, and its SAH distribution fills most of
    their eight child slots."""
    desc, _ = small_sphere_room()
    wide = make_scene(desc, _abi.BVH_DEVICE_WIDE4).bvh_info()
    comp = make_scene(desc, _abi.BVH_DEVICE).bvh_info()
    assert comp["on_device"] == 1 and wide["on_device"] == 1 and comp["num_nodes"] < wide["num_nodes"]
    assert 1 <= comp["stack_bound"] <= 32
    assert comp["inner_children"] == comp["num_nodes"] - 1
    assert (comp["inner_children"] + comp["leaf_children"]) / comp["num_nodes"] > 5.0, comp


def test_large_coordinates_fall_back_to_four_wide_nodes(cuda_device):
    """Coordinates of 1.6e7 and more get 4-wide nodes from the default
    builder, with the same hits as the oracle."""
    desc = scenes.cornell_box()[0]
    desc.positions = (np.asarray(desc.positions, np.float64) * 1e6 + 5e7).astype(np.float32)
    desc.emitter_faces = (np.asarray(desc.emitter_faces, np.float64) * 1e6 + 5e7).astype(np.float32)
    sc = Scene(desc)
    assert sc.bvh_info()["format"] == _abi.BVH_FORMAT_WIDE4
    o = op.Oracle.from_scene(desc, 4, 4, make_params(sc.scene_size), triangles=sc.read_triangles())
    rays = random_rays(desc, 1 << 14, seed=5)
    g, c = gpu_trace(sc, rays, False), o.trace(rays)
    assert (g["prim"] != _abi.INVALID_PRIM).mean() > 0.5
    assert first_mismatch(g, c) is None, first_mismatch(g, c)


@pytest.mark.parametrize("gather_n,gather_m,storage", [(2, 9, _abi.STORAGE_FP32), (3, 5, _abi.STORAGE_FP16),
                                                       (2, 1, _abi.STORAGE_FP32)])
def test_final_gather_with_extra_prefixes(cuda_device, gather_n, gather_m, storage):
    """gatherN > 1 (shader/final_gather.cu:190-321) on the shift machines:
    the extra prefixes continue each pixel's random stream, search at their
    last vertex and add their neighbours' shifted suffixes; with k = 0
    (gatherM = 1) they draw nothing and add zero."""
    desc, cam = small_sphere_room()
    p = large_config_params(scene_size_of(desc), gather_radius=0.3, gather_n=gather_n, gather_m=gather_m,
                            storage=storage, enable_accum=1)
    run_parity(desc, cam, p, 48, 40, 3, lambda c, f: orbit(c, f, 120))
