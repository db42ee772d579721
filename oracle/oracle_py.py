"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the oracle (liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from crisoptix_b200 import _abi  # noqa: E402  (struct layouts of include/crisb.h)

LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("restir_oracle.cpp", "oracle.h", "kat.h", "Makefile")]
    srcs.append(os.path.join(ROOT, "include", "crisb.h"))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs):
        subprocess.run(["make", "-s", "-B" if force else "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = ctypes.CDLL(LIB)
    vp, u32, u64, i32, f32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_float
    sig = {
        "oracle_create": (vp, [vp, vp, vp, u32, vp, u32, vp, u32, vp, u32, u32, u32, ctypes.POINTER(_abi.Params)]),
        "oracle_destroy": (None, [vp]),
        "oracle_set_params": (i32, [vp, ctypes.POINTER(_abi.Params)]),
        "oracle_set_threads": (i32, [i32]),
        "oracle_scene_size": (f32, [vp]),
        "oracle_render_frame": (i32, [vp, ctypes.POINTER(_abi.Camera), vp]),
        "oracle_render_frame_timed": (i32, [vp, ctypes.POINTER(_abi.Camera), vp, vp]),
        "oracle_set_motion_vectors": (i32, [vp, vp, u32]),
        "oracle_set_textures": (i32, [vp, vp, u32, vp, u32, vp]),
        "oracle_tex_sample": (None, [vp, u32, u32, vp, u32, vp]),
        "oracle_frame_index": (u64, [vp]),
        "oracle_frame_random": (u32, [vp]),
        "oracle_dump": (i32, [vp, i32, vp, ctypes.c_size_t]),
        "oracle_check_post_recon": (i32, [vp, ctypes.POINTER(u32), ctypes.POINTER(u32), ctypes.POINTER(u32)]),
        "oracle_dump_size": (ctypes.c_size_t, [vp, i32]),
        "oracle_trace": (i32, [vp, vp, vp, u32, i32]),
        "oracle_trace_bruteforce": (i32, [vp, vp, vp, u32, i32]),
        "oracle_pt_accumulate": (i32, [vp, ctypes.POINTER(_abi.Camera), u32, u64, vp]),
        "oracle_pcg32": (None, [u64, u64, u32, vp]),
        "oracle_tea64": (u64, [u32, u32]),
        "oracle_kat": (i32, [i32, vp, u32, vp]),
        "oracle_oct_unstable": (u64, [vp, u32]),
        "oracle_kat_emitter": (i32, [vp, u32, vp, vp, u32, vp, vp]),
        "oracle_sincos": (None, [vp, u32, vp, vp]),
        "oracle_half": (None, [vp, u32, vp, vp]),
        "oracle_srgb_root": (None, [vp, u32, vp]),
        "oracle_tonemap_srgb8": (i32, [vp, vp, u32]),
        "oracle_srgb8_first_decrease": (u32, [u32, u32]),
        "oracle_oct": (None, [vp, u32, vp, vp]),
        "oracle_camera_data": (i32, [ctypes.POINTER(_abi.Camera), ctypes.POINTER(_abi.CameraData)]),
        "oracle_frame_random_for": (u32, [u64, u64]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def set_threads(n: int) -> int:
    return load().oracle_set_threads(n)


class Oracle:
    """CPU restatement of the frame loop over a world-space triangle soup."""

    def __init__(self, tri_pos, tri_nrm, tri_mat, materials, emitters, emitter_faces, width, height,
                 params: _abi.Params):
        lib = load()
        self.width, self.height = width, height
        self._pos = np.ascontiguousarray(tri_pos, np.float32).reshape(-1, 9)
        self._nrm = np.ascontiguousarray(tri_nrm, np.float32).reshape(-1, 9)
        self._mat = np.ascontiguousarray(tri_mat, np.uint32)
        mats = (_abi.Material * len(materials))()
        for i, m in enumerate(materials):
            mats[i].diffuse[:] = [float(v) for v in m["diffuse"]]
            mats[i].specular[:] = [float(v) for v in m["specular"]]
            mats[i].emission[:] = [float(v) for v in m["emission"]]
            mats[i].roughness = float(m["roughness"])
            mats[i].spec_usage = int(m["spec_usage"])
        ems = (_abi.Emitter * len(emitters))()
        for i, (color, first, count) in enumerate(emitters):
            ems[i].color[:] = [float(v) for v in color]
            ems[i].first_face = int(first)
            ems[i].num_faces = int(count)
        self._faces = np.ascontiguousarray(emitter_faces, np.float32).reshape(-1, 9)
        self._mats, self._ems = mats, ems
        h = lib.oracle_create(_ptr(self._pos), _ptr(self._nrm), _ptr(self._mat), len(self._mat),
                              ctypes.cast(mats, ctypes.c_void_p), len(materials), ctypes.cast(ems, ctypes.c_void_p),
                              len(emitters), _ptr(self._faces), len(self._faces), width, height, ctypes.byref(params))
        if not h:
            raise RuntimeError("oracle_create rejected the scene or parameters")
        self.h = h
        self.storage = int(params.storage)

    @classmethod
    def from_scene(cls, scene_desc, width, height, params, triangles=None):
        """Oracle over a scene description; `triangles` = (pos, nrm, mat) soup
        (defaults to the scene's own float64 flattening)."""
        pos, nrm, mat = triangles if triangles is not None else scene_desc.flatten()
        o = cls(pos, nrm, mat, scene_desc.materials, scene_desc.emitters, scene_desc.emitter_faces, width, height,
                params)
        if getattr(scene_desc, "textured", False):
            o.set_textures(scene_desc.flatten_uvs(), scene_desc.textures, scene_desc.material_textures)
        return o

    def set_textures(self, tri_uvs, textures, material_textures):
        """(T, 6) corner uvs, (H, W, 4) uint8 textures, (M, 3) texture indices."""
        uv = np.ascontiguousarray(tri_uvs, np.float32)
        keep = [np.ascontiguousarray(t, np.uint8) for t in textures]
        tex = (_abi.Texture * max(len(keep), 1))()
        for i, t in enumerate(keep):
            tex[i].rgba = t.ctypes.data_as(ctypes.c_void_p)
            tex[i].height, tex[i].width = int(t.shape[0]), int(t.shape[1])
        mt = np.ascontiguousarray(material_textures, np.int32)
        if load().oracle_set_textures(self.h, _ptr(uv), len(uv), ctypes.cast(tex, ctypes.c_void_p), len(keep),
                                      _ptr(mt)) != 0:
            raise ValueError("oracle rejected the textures")

    def __del__(self):
        if getattr(self, "h", None):
            load().oracle_destroy(self.h)
            self.h = None

    def set_params(self, params):
        if load().oracle_set_params(self.h, ctypes.byref(params)) != 0:
            raise ValueError("oracle rejected parameters")
        self.storage = int(params.storage)

    @property
    def scene_size(self) -> float:
        return load().oracle_scene_size(self.h)

    def set_motion_vectors(self, motion):
        """(H, W, 2) float motion vectors for MOTION_VECTORS (None clears)."""
        if motion is None:
            assert load().oracle_set_motion_vectors(self.h, None, 0) == 0
            return
        m = np.ascontiguousarray(motion, np.float32)
        assert m.size == 2 * self.width * self.height
        assert load().oracle_set_motion_vectors(self.h, _ptr(m), self.width * self.height) == 0

    def render_frame(self, cam, out: np.ndarray, timed: bool = False):
        from crisoptix_b200 import camera_struct
        assert out.dtype == np.float32 and out.size == self.width * self.height * 3 and out.flags.c_contiguous
        c = camera_struct(cam)
        if timed:
            ms = np.zeros(6, np.float64)
            load().oracle_render_frame_timed(self.h, ctypes.byref(c), _ptr(out), _ptr(ms))
            return ms
        if load().oracle_render_frame(self.h, ctypes.byref(c), _ptr(out)) != 0:
            raise ValueError("oracle rejected the frame (motion vectors missing?)")
        return None

    def frame_index(self) -> int:
        return load().oracle_frame_index(self.h)

    def frame_random(self) -> int:
        return load().oracle_frame_random(self.h)

    def dump(self, buffer_id: int) -> np.ndarray:
        n = load().oracle_dump_size(self.h, buffer_id)
        dt = _abi.buffer_dtype(buffer_id, self.storage)
        out = np.zeros(n // dt.itemsize, dtype=dt)
        if n and load().oracle_dump(self.h, buffer_id, _ptr(out), n) != 0:
            raise RuntimeError("oracle_dump failed")
        return out

    def check_post_recon(self) -> dict:
        """oracle_check_post_recon: the front suffix samples re-traced past
        their reconnection vertex from their seeds against their stored
        postReconF (test infrastructure for the resampled-path adjoint)."""
        c, m, n = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        if load().oracle_check_post_recon(self.h, ctypes.byref(c), ctypes.byref(m), ctypes.byref(n)) != 0:
            raise RuntimeError("oracle_check_post_recon failed")
        return {"checked": c.value, "mismatched": m.value, "nee_recon": n.value}

    def trace(self, rays: np.ndarray, any_hit: bool = False, brute: bool = False) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = np.zeros(len(rays), _abi.TRACE_HIT_DTYPE)
        fn = load().oracle_trace_bruteforce if brute else load().oracle_trace
        fn(self.h, _ptr(rays), _ptr(hits), len(rays), 1 if any_hit else 0)
        return hits

    def pt_accumulate(self, cam, spp: int, seed: int, accum: np.ndarray):
        from crisoptix_b200 import camera_struct
        assert accum.dtype == np.float64 and accum.flags.c_contiguous
        load().oracle_pt_accumulate(self.h, ctypes.byref(camera_struct(cam)), spp, seed, _ptr(accum))


def pcg32(initstate: int, initseq: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    load().oracle_pcg32(initstate, initseq, n, _ptr(out))
    return out


def tea64(v0: int, v1: int) -> int:
    return load().oracle_tea64(v0, v1)


def sincos(phi: np.ndarray):
    phi = np.ascontiguousarray(phi, np.float32)
    s = np.zeros_like(phi)
    c = np.zeros_like(phi)
    load().oracle_sincos(_ptr(phi), len(phi), _ptr(s), _ptr(c))
    return s, c


def half(x: np.ndarray):
    """binary16 bits and values of the FP16 storage rule (NaN -> 0, clamp at
    +-65504, round to nearest even)."""
    x = np.ascontiguousarray(x, np.float32)
    bits = np.zeros(x.shape, np.uint16)
    back = np.zeros_like(x)
    load().oracle_half(_ptr(x), x.size, _ptr(bits), _ptr(back))
    return bits, back


def srgb_root(x: np.ndarray) -> np.ndarray:
    """x^(1/2.4) as the sRGB curve computes it (float in, float out)."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros_like(x)
    load().oracle_srgb_root(_ptr(x), x.size, _ptr(out))
    return out


def tonemap_srgb8(rgb: np.ndarray) -> np.ndarray:
    """ToneMapping of (..., 3) linear float RGB to sRGB bytes."""
    x = np.ascontiguousarray(rgb, np.float32)
    assert x.shape[-1] == 3
    out = np.zeros(x.shape, np.uint8)
    assert load().oracle_tonemap_srgb8(_ptr(x), _ptr(out), x.size // 3) == 0
    return out


def srgb8_first_decrease(lo: float, hi: float) -> int:
    """First float bit pattern in (lo, hi] whose byte is below its
    predecessor's (0: the bytes never decrease on [lo, hi])."""
    lo_b = int(np.float32(lo).view(np.uint32))
    hi_b = int(np.float32(hi).view(np.uint32))
    return int(load().oracle_srgb8_first_decrease(lo_b, hi_b))


def tex_sample(rgba: np.ndarray, uv: np.ndarray) -> np.ndarray:
    """The oracle's texture fetch of an (H, W, 4) uint8 texture at (n, 2)
    normalised coordinates: (n, 4) floats."""
    t = np.ascontiguousarray(rgba, np.uint8)
    q = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    out = np.zeros((len(q), 4), np.float32)
    load().oracle_tex_sample(_ptr(t), t.shape[1], t.shape[0], _ptr(q), len(q), _ptr(out))
    return out


def oct(dirs: np.ndarray):
    """Octahedral codes of (n, 3) directions and the decoded unit vectors."""
    d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
    codes = np.zeros(len(d), np.uint32)
    dec = np.zeros_like(d)
    load().oracle_oct(_ptr(d), len(d), _ptr(codes), _ptr(dec))
    return codes, dec


def camera_data(cam) -> np.ndarray:
    from crisoptix_b200 import camera_struct
    d = _abi.CameraData()
    load().oracle_camera_data(ctypes.byref(camera_struct(cam)), ctypes.byref(d))
    return np.array([list(d.pos), list(d.u), list(d.v), list(d.w)], dtype=np.float32)


def frame_random(seed: int, counter: int) -> int:
    return load().oracle_frame_random_for(seed, counter)
