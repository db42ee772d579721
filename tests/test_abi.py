"""The C-ABI library loads and exports what include/crisb.h declares; struct
layouts agree; host-only entry points behave (CPU, no GPU needed)."""
import ctypes
import os
import re

import numpy as np

import oracle_py as op
from crisoptix_b200 import _abi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    src = open(os.path.join(ROOT, "include", "crisb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(crisb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    names = declared_entry_points()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_abi.ENTRY_POINTS), set(names) ^ set(_abi.ENTRY_POINTS)


def test_struct_layouts_match():
    lib = _abi.load()
    n = lib.crisb_abi_sizes(None, 0)
    sizes = (ctypes.c_uint32 * n)()
    lib.crisb_abi_sizes(sizes, n)
    assert n == len(_abi.ABI_STRUCTS)
    for got, t in zip(sizes, _abi.ABI_STRUCTS):
        assert got == _abi.abi_size(t), t


def test_reference_defaults():
    lib = _abi.load()
    p = _abi.Params()
    assert lib.crisb_params_default(ctypes.byref(p), ctypes.c_float(10.0)) == 0
    assert p.nee_prob == np.float32(0.3) and p.max_path_len == 8 and p.prefix_len == 2
    assert abs(p.recon_min_distance - 0.1) < 1e-7 and p.gather_m == 1 and p.window_radius == 10
    assert p.suffix_enable_spatial == 1 and p.prefix_enable_spatial == 0


def test_camera_data_bit_identical_to_oracle():
    lib = _abi.load()
    from crisoptix_b200 import camera_struct
    for k in range(20):
        cam = scenes.orbit_camera(scenes.sphere_room(num_spheres=1, subdiv=0, num_emitters=1)[1], k, 17)
        d = _abi.CameraData()
        assert lib.crisb_camera_get_data(ctypes.byref(camera_struct(cam)), ctypes.byref(d)) == 0
        got = np.array([list(d.pos), list(d.u), list(d.v), list(d.w)], np.float32)
        assert got.tobytes() == op.camera_data(cam).tobytes()


def test_null_arguments_are_rejected_without_a_gpu():
    lib = _abi.load()
    h = ctypes.c_void_p()
    assert lib.crisb_scene_create(None, ctypes.byref(h)) == _abi.ERR_INVALID_ARGUMENT
    buf = ctypes.create_string_buffer(256)
    assert lib.crisb_last_error(buf, 256) == 0 and b"null" in buf.value
    assert lib.crisb_renderer_create(None, 8, 8, None, ctypes.byref(h)) == _abi.ERR_INVALID_ARGUMENT
    assert lib.crisb_render_frame(None, None, None, None) == _abi.ERR_INVALID_ARGUMENT
    # the resampled-path adjoint and the spatial-count tuner
    assert lib.crisb_restir_adjoint_enable(None, 1) == _abi.ERR_INVALID_ARGUMENT
    assert lib.crisb_restir_adjoint_forward(None, None, None) == _abi.ERR_INVALID_ARGUMENT
    assert lib.crisb_restir_adjoint_backward(None, None, None, None, None) == _abi.ERR_INVALID_ARGUMENT
    assert lib.crisb_autotune_spatial(None, None, 1, 1.0, None, None) == _abi.ERR_INVALID_ARGUMENT
