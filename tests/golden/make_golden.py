"""Generate the golden vectors in tests/golden/ from the oracle.

The reference (CrisOptix) cannot run here -- it needs the OptiX SDK and an
OpenGL window -- so the vectors come from the oracle, the CPU restatement of
its frame loop in oracle/.  They pin the oracle and the CUDA path against
silent drift.  Regenerate only for an intended semantic change:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.dirname(HERE)]

import oracle_py as op  # noqa: E402
from crisoptix_b200 import _abi, scenes  # noqa: E402
from helpers import large_config_params, make_params, orbit, scene_size_of, small_config_params, \
    small_sphere_room, static  # noqa: E402

CASES = {
    "cornell_conditional": dict(scene="cornell", W=24, H=20, frames=3, cam="static",
                                params=("small", dict(gather_m=5, gather_radius=0.4))),
    "cornell_pathtracer": dict(scene="cornell", W=16, H=16, frames=2, cam="static",
                               params=("plain", dict(renderer_type=_abi.PATH_TRACER, max_path_len=4))),
    "cornell_restirpt": dict(scene="cornell", W=16, H=16, frames=2, cam="static",
                             params=("plain", dict(renderer_type=_abi.RESTIR_PT, max_path_len=4,
                                                   prefix_enable_spatial=1, prefix_spatial_count=2))),
    "spheres_large_params": dict(scene="spheres", W=24, H=24, frames=3, cam="orbit",
                                 params=("large", dict(gather_radius=0.3))),
    "cornell_textured": dict(scene="cornell_textured", W=24, H=20, frames=3, cam="orbit",
                             params=("small", dict(gather_m=5, gather_radius=0.4))),
    "cornell_reproject": dict(scene="cornell", W=24, H=20, frames=4, cam="orbit",
                              params=("small", dict(motion_mode=_abi.MOTION_REPROJECT))),
    "spheres_fp16": dict(scene="spheres", W=24, H=24, frames=3, cam="orbit",
                         params=("large", dict(gather_radius=0.3, storage=_abi.STORAGE_FP16))),
}

STATE = [_abi.BUF_PREFIX_RES_FRONT, _abi.BUF_CANON_PREFIX, _abi.BUF_SUFFIX_RES_FRONT, _abi.BUF_CANON_SUFFIX,
         _abi.BUF_GBUFFER, _abi.BUF_NEIGHBORS, _abi.BUF_NEIGHBOR_COUNT]


def case_inputs(case):
    desc, cam = {"cornell": scenes.cornell_box, "cornell_textured": scenes.textured_cornell_box,
                 "spheres": small_sphere_room}[case["scene"]]()
    kind, kw = case["params"]
    size = scene_size_of(desc)
    p = {"small": small_config_params, "large": large_config_params, "plain": make_params}[kind](size, **kw)
    cam_fn = static if case["cam"] == "static" else (lambda c, f: orbit(c, f, 120))
    return desc, cam, p, cam_fn


def run_oracle(case, triangles=None):
    desc, cam, p, cam_fn = case_inputs(case)
    o = op.Oracle.from_scene(desc, case["W"], case["H"], p, triangles=triangles)
    out = np.zeros((case["H"], case["W"], 3), np.float32)
    for f in range(case["frames"]):
        o.render_frame(cam_fn(cam, f), out)
    return out, {str(b): o.dump(b) for b in STATE}


def main(names=None):
    for name, case in CASES.items():
        if names and name not in names:
            continue
        img, state = run_oracle(case)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), image=img,
                            **{"buf" + k: v.view(np.uint8) for k, v in state.items()})
        print(name, img.mean())


if __name__ == "__main__":
    main(sys.argv[1:])
