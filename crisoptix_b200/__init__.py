"""crisoptix_b200 -- B200-native Conditional ReSTIR PT frame loop.

Python view of the C ABI in include/crisb.h, shaped like the reference's host
API: ``Scene`` (include/model/Scene.h:12-24), ``Renderer``
(include/graph/Renderer.h:11-21) with ``launch_frame`` / ``get_frame_idx``,
and a camera description (include/graph/Camera.h).  All compute runs in the
in-tree CUDA library libcrisb.so; importing works without a GPU, creating a
scene or renderer needs one.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _abi
from ._abi import CrisbError, check, load
from .scenes import Camera as CameraDesc
from .scenes import Scene as SceneDesc

__all__ = ["Scene", "Renderer", "Batch", "CameraDesc", "SceneDesc", "default_params", "camera_struct", "CrisbError",
           "load"]


def camera_struct(cam: CameraDesc) -> _abi.Camera:
    c = _abi.Camera()
    c.pos[:] = cam.pos
    c.view_dir[:] = cam.view_dir
    c.up[:] = cam.up
    c.aspect = cam.aspect
    c.fov = cam.fov
    c.changed = 1 if cam.changed else 0
    return c


def camera_data(cam: CameraDesc) -> np.ndarray:
    """Camera::GetData -> (pos, U, V, W) as a (4, 3) float32 array."""
    d = _abi.CameraData()
    check(load().crisb_camera_get_data(ctypes.byref(camera_struct(cam)), ctypes.byref(d)))
    return np.array([list(d.pos), list(d.u), list(d.v), list(d.w)], dtype=np.float32)


def default_params(scene_size: float, **overrides) -> _abi.Params:
    """Renderer defaults of src/Renderer.cpp:34-58, then `overrides`."""
    p = _abi.Params()
    check(load().crisb_params_default(ctypes.byref(p), ctypes.c_float(scene_size)))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class Scene:
    """Scene(instances, emitters): flattens instances and builds the BVH of
    the current CUDA device (on the device into compressed 8-wide nodes by
    default; builder=BVH_DEVICE_WIDE4 builds 4-wide nodes on the device,
    BVH_HOST 4-wide nodes on the host)."""

    def __init__(self, desc: SceneDesc, builder: int = _abi.BVH_DEVICE):
        lib = load()
        self.desc = desc
        self._keep = []

        def arr(a, dtype):
            a = np.ascontiguousarray(a, dtype=dtype)
            self._keep.append(a)
            return a.ctypes.data_as(ctypes.c_void_p)

        d = _abi.SceneDesc()
        d.positions = arr(desc.positions, np.float32)
        d.normals = arr(desc.normals, np.float32)
        d.num_vertices = len(desc.positions)
        d.indices = arr(desc.indices, np.uint32)
        d.triangle_material = arr(desc.triangle_material, np.uint32)
        d.num_triangles = len(desc.indices)
        mats = (_abi.Material * len(desc.materials))()
        for i, m in enumerate(desc.materials):
            mats[i].diffuse[:] = [float(v) for v in m["diffuse"]]
            mats[i].specular[:] = [float(v) for v in m["specular"]]
            mats[i].emission[:] = [float(v) for v in m["emission"]]
            mats[i].roughness = float(m["roughness"])
            mats[i].spec_usage = int(m["spec_usage"])
        self._keep.append(mats)
        d.materials = ctypes.cast(mats, ctypes.c_void_p)
        d.num_materials = len(desc.materials)
        if desc.instances:
            meshes = (_abi.Mesh * len(desc.meshes))()
            for i, (f, n) in enumerate(desc.meshes):
                meshes[i].first_triangle = int(f)
                meshes[i].num_triangles = int(n)
            inst = (_abi.Instance * len(desc.instances))()
            for i, (m, ov, xf) in enumerate(desc.instances):
                inst[i].mesh = int(m)
                inst[i].material_override = int(ov)
                inst[i].transform[:] = [float(v) for v in xf]
            self._keep += [meshes, inst]
            d.meshes = ctypes.cast(meshes, ctypes.c_void_p)
            d.num_meshes = len(desc.meshes)
            d.instances = ctypes.cast(inst, ctypes.c_void_p)
            d.num_instances = len(desc.instances)
        ems = (_abi.Emitter * len(desc.emitters))()
        for i, (color, first, count) in enumerate(desc.emitters):
            ems[i].color[:] = [float(v) for v in color]
            ems[i].first_face = int(first)
            ems[i].num_faces = int(count)
        self._keep.append(ems)
        d.emitters = ctypes.cast(ems, ctypes.c_void_p)
        d.num_emitters = len(desc.emitters)
        d.emitter_faces = arr(desc.emitter_faces, np.float32)
        d.num_emitter_faces = len(desc.emitter_faces)
        d.bvh_builder = int(builder)
        if desc.material_textures is not None:
            mt = np.ascontiguousarray(desc.material_textures, np.int32)
            if mt.shape != (len(desc.materials), 3):
                raise ValueError("material_textures must be (num_materials, 3)")
            d.material_textures = arr(mt, np.int32)
            if desc.uvs is not None:
                d.uvs = arr(desc.uvs, np.float32)
            tex = (_abi.Texture * max(len(desc.textures), 1))()
            for i, t in enumerate(desc.textures):
                t = np.ascontiguousarray(t, np.uint8)
                if t.ndim != 3 or t.shape[2] != 4:
                    raise ValueError("textures must be (H, W, 4) uint8")
                tex[i].rgba = arr(t, np.uint8)
                tex[i].height, tex[i].width = int(t.shape[0]), int(t.shape[1])
            self._keep.append(tex)
            d.textures = ctypes.cast(tex, ctypes.c_void_p)
            d.num_textures = len(desc.textures)
        h = ctypes.c_void_p()
        check(lib.crisb_scene_create(ctypes.byref(d), ctypes.byref(h)))
        self.handle = h
        self._keep.clear()

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                load().crisb_scene_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None

    @property
    def scene_size(self) -> float:
        v = ctypes.c_float()
        check(load().crisb_scene_size(self.handle, ctypes.byref(v)))
        return v.value

    @property
    def num_triangles(self) -> int:
        v = ctypes.c_uint32()
        check(load().crisb_scene_num_triangles(self.handle, ctypes.byref(v)))
        return v.value

    def bvh_info(self) -> dict:
        """The BVH as built: format (BVH_FORMAT_*), on_device, num_nodes,
        node_bytes, stack_bound, depth, inner_children, leaf_children."""
        v = _abi.BvhInfo()
        check(load().crisb_scene_bvh_info(self.handle, ctypes.byref(v)))
        return {k: getattr(v, k) for k, _ in _abi.BvhInfo._fields_}

    def read_triangles(self):
        """World-space triangle soup: (T, 9) positions, (T, 9) normals, (T,)
        materials, in scene order."""
        n = self.num_triangles
        pos = np.zeros((n, 9), np.float32)
        nrm = np.zeros((n, 9), np.float32)
        mat = np.zeros(n, np.uint32)
        check(load().crisb_scene_read_triangles(self.handle, pos.ctypes.data_as(ctypes.c_void_p),
                                                 nrm.ctypes.data_as(ctypes.c_void_p),
                                                 mat.ctypes.data_as(ctypes.c_void_p)))
        return pos, nrm, mat

    def trace(self, rays_dev_ptr: int, hits_dev_ptr: int, n: int, any_hit: bool, stream: int = 0):
        check(load().crisb_trace_rays(self.handle, ctypes.c_void_p(rays_dev_ptr), ctypes.c_void_p(hits_dev_ptr),
                                      n, 1 if any_hit else 0, ctypes.c_void_p(stream)))


class Renderer:
    """Renderer(width, height, camera, scene): the Conditional ReSTIR PT
    frame loop on the scene's device."""

    def __init__(self, width: int, height: int, scene: Scene, params: Optional[_abi.Params] = None):
        self.scene = scene
        self.width = width
        self.height = height
        if params is None:
            params = default_params(scene.scene_size)
        h = ctypes.c_void_p()
        check(load().crisb_renderer_create(scene.handle, width, height, ctypes.byref(params), ctypes.byref(h)))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                load().crisb_renderer_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None

    @property
    def params(self) -> _abi.Params:
        p = _abi.Params()
        check(load().crisb_renderer_get_params(self.handle, ctypes.byref(p)))
        return p

    @params.setter
    def params(self, p: _abi.Params):
        check(load().crisb_renderer_set_params(self.handle, ctypes.byref(p)))

    def launch_frame(self, camera: CameraDesc, out_dev_ptr: int, stream: int = 0):
        """Renderer::LaunchFrame into a device buffer of width*height*3 floats."""
        check(load().crisb_render_frame(self.handle, ctypes.byref(camera_struct(camera)), ctypes.c_void_p(out_dev_ptr),
                                        ctypes.c_void_p(stream)))

    def restir_adjoint_enable(self, on: bool = True):
        """From the next frame on, keep what the resampled-path adjoint reads
        (crisb_restir_adjoint_enable)."""
        check(load().crisb_restir_adjoint_enable(self.handle, 1 if on else 0))

    def restir_adjoint_forward(self, out_dev_ptr: int, stream: int = 0):
        """The last frame's final-gather estimator at the scene's current
        tables, frozen at the frame's (width*height*3 floats)."""
        check(load().crisb_restir_adjoint_forward(self.handle, ctypes.c_void_p(out_dev_ptr), ctypes.c_void_p(stream)))

    def restir_adjoint_backward(self, d_img_ptr: int, d_mats_ptr: int, d_em_ptr: int, stream: int = 0):
        """Adds dLoss/dparameter of the last frame's final-gather estimator
        (7 floats per material, 3 per emitter) for d_img = dLoss/dimage."""
        check(load().crisb_restir_adjoint_backward(self.handle, ctypes.c_void_p(d_img_ptr), ctypes.c_void_p(d_mats_ptr),
                                                   ctypes.c_void_p(d_em_ptr), ctypes.c_void_p(stream)))

    def get_frame_idx(self) -> int:
        v = ctypes.c_uint64()
        check(load().crisb_frame_index(self.handle, ctypes.byref(v)))
        return v.value

    def frame_random(self) -> int:
        v = ctypes.c_uint32()
        check(load().crisb_frame_random(self.handle, ctypes.byref(v)))
        return v.value

    def set_trace_grid(self, blocks_per_resident_block: int):
        check(load().crisb_set_trace_grid(self.handle, int(blocks_per_resident_block)))

    def autotune(self, camera: CameraDesc, frames: int = 3) -> dict:
        """Pick the launch settings (traversal block size and grid, job
        capacity) by timing candidates on a scratch renderer (this renderer's
        state is untouched); applies and returns the choices."""
        t = _abi.Tuning()
        check(load().crisb_autotune_ex(self.handle, ctypes.byref(camera_struct(camera)), int(frames), ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def autotune_spatial(self, camera: CameraDesc, budget_ms: float, frames: int = 3) -> dict:
        """Pick suffix_spatial_count for a frame budget (crisb_autotune_spatial):
        the largest candidate count whose frame time fits; applies it and
        returns {"count", "frame_ms"}.  Changes the estimator."""
        c, ms = ctypes.c_uint32(), ctypes.c_float()
        check(load().crisb_autotune_spatial(self.handle, ctypes.byref(camera_struct(camera)), int(frames),
                                            ctypes.c_float(budget_ms), ctypes.byref(c), ctypes.byref(ms)))
        return {"count": c.value, "frame_ms": ms.value}

    def set_trace_block(self, threads: int):
        check(load().crisb_set_trace_block(self.handle, int(threads)))

    def set_motion_vectors(self, motion_dev_ptr: int):
        """width * height float pairs on the device for MOTION_VECTORS (0 clears)."""
        check(load().crisb_set_motion_vectors(self.handle, motion_dev_ptr or None))

    def set_srgb_output(self, srgb_dev_ptr: int):
        """Tone-map each frame into width * height * 3 device bytes (0 stops)."""
        check(load().crisb_set_srgb_output(self.handle, srgb_dev_ptr or None))

    def set_job_capacity(self, jobs_per_pixel: int):
        """Shift-machine job records per pixel (memory against speed; results
        do not depend on it)."""
        check(load().crisb_set_job_capacity(self.handle, int(jobs_per_pixel)))

    def job_capacity(self) -> int:
        v = ctypes.c_uint32()
        check(load().crisb_get_job_capacity(self.handle, ctypes.byref(v)))
        return v.value

    def set_graph(self, enable: bool):
        """Run frames as one CUDA graph of the pass chain (default) or launch
        the kernels directly; the results are identical."""
        check(load().crisb_set_graph(self.handle, 1 if enable else 0))

    def set_timing(self, level: int):
        """0 off, 1 per-pass / per-kernel-class CUDA events, 2 also ray counters."""
        check(load().crisb_set_timing(self.handle, int(level)))

    def stats(self) -> dict:
        s = _abi.Stats()
        check(load().crisb_get_stats(self.handle, ctypes.byref(s)))
        d = {k: getattr(s, k) for k, _ in s._fields_ if k != "resample_bytes"}
        d["resample_bytes"] = dict(zip(_abi.RESAMPLE_KERNELS, (int(v) for v in s.resample_bytes)))
        return d

    def check_device_errors(self):
        check(load().crisb_check_device_errors(self.handle))

    def debug_read(self, buffer_id: int) -> np.ndarray:
        size = ctypes.c_size_t()
        check(load().crisb_debug_size(self.handle, buffer_id, ctypes.byref(size)))
        dt = _abi.buffer_dtype(buffer_id, self.params.storage)
        out = np.zeros(size.value // dt.itemsize, dtype=dt)
        check(load().crisb_debug_read(self.handle, buffer_id, out.ctypes.data_as(ctypes.c_void_p), size.value))
        return out


class Batch:
    """Several renderers (views) of one device whose frames run as parallel
    branches of one CUDA graph (include/crisb.h, crisb_batch_render)."""

    def __init__(self, renderers):
        self.renderers = list(renderers)
        arr = (ctypes.c_void_p * len(self.renderers))(*[r.handle.value for r in self.renderers])
        h = ctypes.c_void_p()
        check(load().crisb_batch_create(arr, len(self.renderers), ctypes.byref(h)))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                load().crisb_batch_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None

    def render(self, cameras, out_dev_ptrs, stream: int = 0):
        """One frame of every view: cameras[k] into the device buffer
        out_dev_ptrs[k] (W*H*3 floats of renderer k)."""
        n = len(self.renderers)
        if len(cameras) != n or len(out_dev_ptrs) != n:
            raise ValueError("one camera and one output per view")
        cams = (_abi.Camera * n)(*[camera_struct(c) for c in cameras])
        outs = (ctypes.c_void_p * n)(*out_dev_ptrs)
        check(load().crisb_batch_render(self.handle, ctypes.cast(cams, ctypes.c_void_p), outs, ctypes.c_void_p(stream)))
