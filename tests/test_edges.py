"""Edge cases of the frame loop against the oracle: tiny and ragged
resolutions, parameter limits, NEE probabilities 0 and 1, accumulation, and a
scene that is nothing but its emitter.  CPU: the oracle itself runs every
case (finite images, no invalid records); GPU: the library bit for bit."""
import numpy as np
import pytest

import oracle_py as op
from crisoptix_b200 import _abi, scenes
from helpers import large_config_params, orbit, scene_size_of, small_config_params, small_sphere_room, static

RESOLUTIONS = [(1, 1), (1, 7), (9, 1), (3, 2), (129, 3), (31, 17)]


def _cases():
    """(id, scene builder, params overrides, W, H, frames, camera path)."""
    cases = []
    for w, h in RESOLUTIONS:
        cases.append((f"res{w}x{h}", "cornell", {}, w, h, 3, "static"))
    cases += [
        ("k31_radius_large", "cornell", dict(gather_m=32, gather_radius=2.0), 24, 20, 2, "static"),
        ("spatial16_3rounds", "cornell", dict(suffix_spatial_count=16, suffix_spatial_rounds=3), 24, 20, 3,
         "orbit"),
        ("window0", "cornell", dict(window_radius=0, suffix_spatial_count=4), 24, 20, 3, "static"),
        ("prefix_len_eq_max", "cornell", dict(max_path_len=3, prefix_len=3), 24, 20, 3, "static"),
        ("max_path_len1", "cornell", dict(max_path_len=1, prefix_len=1), 24, 20, 3, "static"),
        ("nee0", "cornell", dict(nee_prob=0.0), 24, 20, 3, "orbit"),
        ("nee1", "cornell", dict(nee_prob=1.0), 24, 20, 3, "orbit"),
        ("accum", "cornell", dict(enable_accum=1), 24, 20, 4, "static"),
        ("no_temporal", "cornell", dict(prefix_enable_temporal=0, suffix_enable_temporal=0), 24, 20, 3, "static"),
        ("no_spatial", "cornell", dict(suffix_enable_spatial=0), 24, 20, 3, "static"),
        ("emitter_only", "emitter", {}, 16, 16, 3, "static"),
        ("emitter_only_pt", "emitter", dict(renderer_type=_abi.PATH_TRACER), 16, 16, 3, "static"),
        ("emitter_only_restirpt", "emitter", dict(renderer_type=_abi.RESTIR_PT), 16, 16, 3, "static"),
        ("deep_paths", "spheres", dict(max_path_len=16, prefix_len=4), 32, 24, 3, "orbit"),
    ]
    return cases


CASES = _cases()


def _emitter_only():
    """A single emissive quad seen from the front: every path ends at the
    first hit or escapes."""
    desc, cam = scenes.cornell_box()
    b = scenes._Builder()
    b.quad((-0.3, 0.2, 0.0), (0.3, 0.2, 0.0), (0.3, 0.8, 0.0), (-0.3, 0.8, 0.0), 0, (0, 0, 1))
    P, N, idx, tm = b.arrays()
    mats = np.stack([scenes._material((0.5, 0.5, 0.5), emission=(3.0, 2.0, 1.0))])
    faces = P.reshape(2, 9).astype(np.float32)
    s = scenes.Scene(P, N, idx, tm, mats, np.zeros((0, 2), np.uint32), [], [((3.0, 2.0, 1.0), 0, 2)], faces,
                     name="emitter_only")
    return s, cam


def _setup(case):
    name, which, kw, w, h, frames, path = case
    if which == "cornell":
        desc, cam = scenes.cornell_box()
        p = small_config_params(scene_size_of(desc), **kw)
    elif which == "emitter":
        desc, cam = _emitter_only()
        p = small_config_params(scene_size_of(desc), **kw)
    else:
        desc, cam = small_sphere_room()
        p = large_config_params(scene_size_of(desc), gather_radius=0.3, **kw)
    cam_fn = static if path == "static" else (lambda c, f: orbit(c, f, 30))
    return desc, cam, p, w, h, frames, cam_fn


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_runs_edge_case(case):
    desc, cam, p, w, h, frames, cam_fn = _setup(case)
    o = op.Oracle.from_scene(desc, w, h, p)
    out = np.zeros((h, w, 3), np.float32)
    for f in range(frames):
        o.render_frame(cam_fn(cam, f), out)
        assert np.isfinite(out).all()
    if case[0] == "emitter_only":
        # ConditionalRestir does not add emission at the primary vertex
        assert out.max() == 0.0
    if case[0] == "emitter_only_pt":
        assert out.max() == 3.0  # the emitter seen directly, nothing else lit


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_edge_case_parity(cuda_device, case):
    from test_parity_gpu import run_parity

    desc, cam, p, w, h, frames, cam_fn = _setup(case)
    run_parity(desc, cam, p, w, h, frames, cam_fn)
