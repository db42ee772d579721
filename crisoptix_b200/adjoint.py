"""Path-replay adjoints (include/crisb.h): of the path tracer
(crisb_adjoint_*) and of the final gather's resampled estimator
(crisb_restir_adjoint_*).

``PtAdjoint`` and ``RestirAdjoint`` wrap the C ABI; ``PtImage`` and
``RestirImage`` are ``torch.autograd.Function`` classes over them, for checking
only (the library itself needs no torch); ``fd_check`` and
``restir_fd_check`` compare an adjoint's gradient of an L2 image loss with
central differences of the same frozen estimator, summed in float64.

Parameters as the inverse-rendering config names them: per material the
diffuse albedo (3) and roughness (1); per emitter its radiance (3), which the
library holds twice -- the emitter table colour used by next-event estimation
and the emission of the emitter's material seen by camera rays -- so its
gradient is the sum of both.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from ._abi import check, load
from .scenes import MATERIAL_DTYPE, Camera

MAT_GRAD = 7  # diffuse rgb, roughness, emission rgb
EM_GRAD = 3


def get_materials(scene) -> np.ndarray:
    n = len(scene.desc.materials)
    out = np.zeros(n, MATERIAL_DTYPE)
    check(load().crisb_scene_get_materials(scene.handle, out.ctypes.data_as(ctypes.c_void_p), n))
    return out


def set_materials(scene, mats: np.ndarray):
    mats = np.ascontiguousarray(mats, MATERIAL_DTYPE)
    check(load().crisb_scene_set_materials(scene.handle, mats.ctypes.data_as(ctypes.c_void_p), len(mats)))


def set_emitter_colors(scene, rgb: np.ndarray):
    rgb = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    check(load().crisb_scene_set_emitter_colors(scene.handle, rgb.ctypes.data_as(ctypes.c_void_p), len(rgb)))


class PtAdjoint:
    """Frozen-sampling path tracer of `scene` at W x H and its adjoint."""

    def __init__(self, scene, width: int, height: int, params: _abi.Params):
        from . import camera_struct  # noqa: F401  (import check)

        self.scene, self.width, self.height = scene, width, height
        self.num_mats = len(scene.desc.materials)
        self.num_emitters = len(scene.desc.emitters)
        h = ctypes.c_void_p()
        check(load().crisb_adjoint_create(scene.handle, width, height, ctypes.byref(params), ctypes.byref(h)))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                load().crisb_adjoint_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None

    def refreeze(self):
        check(load().crisb_adjoint_refreeze(self.handle))

    def forward(self, cam: Camera, frame: int, out_ptr: int, stream: int = 0):
        from . import camera_struct

        check(load().crisb_adjoint_forward(self.handle, ctypes.byref(camera_struct(cam)), frame,
                                           ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream)))

    def backward(self, cam: Camera, frame: int, d_img_ptr: int, d_mats_ptr: int, d_em_ptr: int, stream: int = 0):
        from . import camera_struct

        check(load().crisb_adjoint_backward(self.handle, ctypes.byref(camera_struct(cam)), frame,
                                            ctypes.c_void_p(d_img_ptr), ctypes.c_void_p(d_mats_ptr),
                                            ctypes.c_void_p(d_em_ptr), ctypes.c_void_p(stream)))

    def render(self, cams: Sequence[Camera], frame: int = 0):
        """(V, H, W, 3) float32 device tensor of every camera's image."""
        import torch

        out = torch.zeros(len(cams), self.height * self.width * 3, dtype=torch.float32, device="cuda")
        for v, c in enumerate(cams):
            self.forward(c, frame, out[v].data_ptr())
        return out.view(len(cams), self.height, self.width, 3)

    def gradient(self, cams: Sequence[Camera], d_img, frame: int = 0, dist=None):
        """(materials x 7, emitters x 3) float32 device tensors of dLoss/dparameter
        for d_img = dLoss/dimage of shape (V, H, W, 3); with a process group
        `dist`, summed over the ranks (each differentiating its own views)."""
        import torch

        from .sharding import sum_gradients

        d_img = d_img.contiguous().view(len(cams), -1).float()
        g_mat = torch.zeros(self.num_mats * MAT_GRAD, dtype=torch.float32, device="cuda")
        g_em = torch.zeros(self.num_emitters * EM_GRAD, dtype=torch.float32, device="cuda")
        for v, c in enumerate(cams):
            self.backward(c, frame, d_img[v].data_ptr(), g_mat.data_ptr(), g_em.data_ptr())
        sum_gradients(g_mat, g_em, dist)
        return g_mat.view(self.num_mats, MAT_GRAD), g_em.view(self.num_emitters, EM_GRAD)


def _apply(scene, base: np.ndarray, diffuse, roughness, emission, emitter_rgb):
    mats = base.copy()
    mats["diffuse"] = diffuse
    mats["roughness"] = roughness
    mats["emission"] = emission
    set_materials(scene, mats)
    set_emitter_colors(scene, emitter_rgb)


def pt_image_function():
    """The torch.autograd.Function class (built lazily so importing this module
    needs no torch)."""
    import torch

    class PtImage(torch.autograd.Function):
        """images = PtImage.apply(diffuse (M,3), roughness (M,), emission (M,3),
        emitter_rgb (E,3), adjoint, base_materials, cameras, frame)"""

        @staticmethod
        def forward(ctx, diffuse, roughness, emission, emitter_rgb, adj, base, cams, frame):
            _apply(adj.scene, base, diffuse.detach().cpu().numpy(), roughness.detach().cpu().numpy(),
                   emission.detach().cpu().numpy(), emitter_rgb.detach().cpu().numpy())
            ctx.adj, ctx.cams, ctx.frame = adj, cams, frame
            ctx.like = (diffuse, roughness, emission, emitter_rgb)
            return adj.render(cams, frame)

        @staticmethod
        def backward(ctx, grad_img):
            g_mat, g_em = ctx.adj.gradient(ctx.cams, grad_img, ctx.frame)
            grads = (g_mat[:, 0:3], g_mat[:, 3], g_mat[:, 4:7], g_em)
            return tuple(g.to(device=t.device, dtype=t.dtype) for g, t in zip(grads, ctx.like)) + (None,) * 4

    return PtImage


class RestirAdjoint:
    """Path-replay adjoint of the resampled estimator over one Conditional
    ReSTIR renderer per view (FP32 storage, gather_n 1, no accumulation).
    ``prepare`` renders `frames` frames of every view at the scene's current
    tables (temporal and spatial reuse fill the reservoirs); ``render`` and
    ``gradient`` then evaluate and differentiate each view's last frame."""

    def __init__(self, scene, width: int, height: int, params: _abi.Params, num_views: int):
        from . import Renderer

        self.scene, self.width, self.height = scene, width, height
        self.num_mats = len(scene.desc.materials)
        self.num_emitters = len(scene.desc.emitters)
        self.views = [Renderer(width, height, scene, params) for _ in range(num_views)]
        for r in self.views:
            r.restir_adjoint_enable(True)
        self.frame_images = None

    def prepare(self, cams: Sequence[Camera], frames: int = 3):
        """Renders the frames; returns the last frame's (V, H, W, 3) images."""
        import torch

        out = torch.zeros(len(cams), self.height * self.width * 3, dtype=torch.float32, device="cuda")
        for f in range(frames):
            for r, c, o in zip(self.views, cams, out):
                r.launch_frame(c, o.data_ptr())
        torch.cuda.synchronize()
        self.frame_images = out.view(len(cams), self.height, self.width, 3)
        return self.frame_images

    def render(self):
        """(V, H, W, 3) float32 device tensor: each view's frozen estimator at
        the scene's current tables."""
        import torch

        out = torch.zeros(len(self.views), self.height * self.width * 3, dtype=torch.float32, device="cuda")
        for r, o in zip(self.views, out):
            r.restir_adjoint_forward(o.data_ptr())
        return out.view(len(self.views), self.height, self.width, 3)

    def gradient(self, d_img, dist=None):
        """(materials x 7, emitters x 3) float32 device tensors of dLoss/dparameter
        for d_img = dLoss/dimage of shape (V, H, W, 3); with a process group
        `dist`, summed over the ranks (each differentiating its own views)."""
        import torch

        from .sharding import sum_gradients

        d_img = d_img.contiguous().view(len(self.views), -1).float()
        g_mat = torch.zeros(self.num_mats * MAT_GRAD, dtype=torch.float32, device="cuda")
        g_em = torch.zeros(self.num_emitters * EM_GRAD, dtype=torch.float32, device="cuda")
        for v, r in enumerate(self.views):
            r.restir_adjoint_backward(d_img[v].data_ptr(), g_mat.data_ptr(), g_em.data_ptr())
        sum_gradients(g_mat, g_em, dist)
        return g_mat.view(self.num_mats, MAT_GRAD), g_em.view(self.num_emitters, EM_GRAD)


def restir_image_function():
    """The torch.autograd.Function class of the resampled estimator (built
    lazily so importing this module needs no torch)."""
    import torch

    class RestirImage(torch.autograd.Function):
        """images = RestirImage.apply(diffuse (M,3), roughness (M,), emission
        (M,3), emitter_rgb (E,3), adjoint, base_materials): the frozen
        estimator of the adjoint's prepared frames at these parameters"""

        @staticmethod
        def forward(ctx, diffuse, roughness, emission, emitter_rgb, adj, base):
            _apply(adj.scene, base, diffuse.detach().cpu().numpy(), roughness.detach().cpu().numpy(),
                   emission.detach().cpu().numpy(), emitter_rgb.detach().cpu().numpy())
            ctx.adj = adj
            ctx.like = (diffuse, roughness, emission, emitter_rgb)
            return adj.render()

        @staticmethod
        def backward(ctx, grad_img):
            g_mat, g_em = ctx.adj.gradient(grad_img)
            grads = (g_mat[:, 0:3], g_mat[:, 3], g_mat[:, 4:7], g_em)
            return tuple(g.to(device=t.device, dtype=t.dtype) for g, t in zip(grads, ctx.like)) + (None,) * 2

    return RestirImage


@dataclass
class Param:
    kind: str   # "diffuse", "roughness" or "radiance"
    index: int  # material (diffuse, roughness) or emitter (radiance)
    channel: int = 0


def emitter_materials(scene_desc) -> List[int]:
    """Material of each emitter's faces (the emission camera rays see)."""
    mats = scene_desc.triangle_material
    faces = np.asarray(scene_desc.emitter_faces, np.float32).reshape(-1, 9)
    P = np.asarray(scene_desc.positions, np.float32)[np.asarray(scene_desc.indices)].reshape(-1, 9)
    out = []
    for color, first, count in scene_desc.emitters:
        hit = np.nonzero(np.all(np.abs(P - faces[first]) < 1e-6, axis=1))[0]
        out.append(int(mats[hit[0]]) if len(hit) else -1)
    return out


def gather(g_mat: np.ndarray, g_em: np.ndarray, params: Sequence[Param], em_mats: Sequence[int]) -> np.ndarray:
    out = np.zeros(len(params), np.float64)
    for k, p in enumerate(params):
        if p.kind == "diffuse":
            out[k] = g_mat[p.index, p.channel]
        elif p.kind == "roughness":
            out[k] = g_mat[p.index, 3]
        else:
            out[k] = g_em[p.index, p.channel]
            if em_mats[p.index] >= 0:
                out[k] += g_mat[em_mats[p.index], 4 + p.channel]
    return out


def perturb(mats: np.ndarray, emitter_rgb: np.ndarray, p: Param, delta: float, em_mats: Sequence[int]):
    mats, emitter_rgb = mats.copy(), emitter_rgb.copy()
    if p.kind == "diffuse":
        mats["diffuse"][p.index, p.channel] += delta
    elif p.kind == "roughness":
        mats["roughness"][p.index] += delta
    else:
        emitter_rgb[p.index, p.channel] += delta
        if em_mats[p.index] >= 0:
            mats["emission"][em_mats[p.index], p.channel] += delta
    return mats, emitter_rgb


def value_of(mats: np.ndarray, emitter_rgb: np.ndarray, p: Param) -> float:
    if p.kind == "diffuse":
        return float(mats["diffuse"][p.index, p.channel])
    if p.kind == "roughness":
        return float(mats["roughness"][p.index])
    return float(emitter_rgb[p.index, p.channel])


def fd_check(scene, desc, cams: Sequence[Camera], width: int, height: int, params: _abi.Params,
             target_mats: np.ndarray, target_rgb: np.ndarray, start_mats: np.ndarray, start_rgb: np.ndarray,
             check_params: Sequence[Param], eps: float = 1e-3, frame: int = 0) -> dict:
    """Adjoint gradient of loss = sum over pixels of (image - target)^2 at the
    start parameters against central differences (relative step `eps`, float64
    loss sums) of the same frozen-sampling estimator, for `check_params`."""
    import torch

    em_mats = emitter_materials(desc)
    set_materials(scene, start_mats)
    set_emitter_colors(scene, start_rgb)
    adj = PtAdjoint(scene, width, height, params)  # sampling frozen at the start parameters
    set_materials(scene, target_mats)
    set_emitter_colors(scene, target_rgb)
    target = adj.render(cams, frame).double()
    set_materials(scene, start_mats)
    set_emitter_colors(scene, start_rgb)
    img = adj.render(cams, frame)
    d_img = 2.0 * (img.double() - target)
    g_mat, g_em = adj.gradient(cams, d_img.float(), frame)
    grad = gather(g_mat.cpu().numpy().astype(np.float64), g_em.cpu().numpy().astype(np.float64), check_params,
                  em_mats)

    def loss(mats, rgb):
        set_materials(scene, mats)
        set_emitter_colors(scene, rgb)
        return float(((adj.render(cams, frame).double() - target) ** 2).sum())

    fd = np.zeros(len(check_params))
    for k, p in enumerate(check_params):
        h = eps * max(abs(value_of(start_mats, start_rgb, p)), 1e-2)
        mp, rp = perturb(start_mats, start_rgb, p, h, em_mats)
        mm, rm = perturb(start_mats, start_rgb, p, -h, em_mats)
        fd[k] = (loss(mp, rp) - loss(mm, rm)) / (2.0 * h)
    set_materials(scene, start_mats)
    set_emitter_colors(scene, start_rgb)
    scale = np.maximum(np.abs(fd), 1e-12)
    rel = np.abs(grad - fd) / scale
    return {"adjoint": grad, "fd": fd, "rel_err": rel, "loss": loss(start_mats, start_rgb)}


def restir_fd_check(scene, desc, cams: Sequence[Camera], width: int, height: int, params: _abi.Params,
                    target_mats: np.ndarray, target_rgb: np.ndarray, start_mats: np.ndarray, start_rgb: np.ndarray,
                    check_params: Sequence[Param], eps: float = 1e-3, frames: int = 3) -> dict:
    """As ``fd_check`` for the resampled estimator: `frames` Conditional ReSTIR
    frames per view at the start parameters, then the adjoint gradient of loss
    = sum of (image - target)^2 (target: the frozen estimator at the target
    parameters) against central differences of the frozen estimator.  Also
    the largest difference between the frozen estimator at the start
    parameters and the frames' own images."""
    em_mats = emitter_materials(desc)
    set_materials(scene, start_mats)
    set_emitter_colors(scene, start_rgb)
    adj = RestirAdjoint(scene, width, height, params, len(cams))
    frame_img = adj.prepare(cams, frames).double()
    start_img = adj.render()
    frame_diff = float((start_img.double() - frame_img).abs().max())
    frame_scale = float(frame_img.abs().max())
    set_materials(scene, target_mats)
    set_emitter_colors(scene, target_rgb)
    target = adj.render().double()
    set_materials(scene, start_mats)
    set_emitter_colors(scene, start_rgb)
    img = adj.render()
    d_img = 2.0 * (img.double() - target)
    g_mat, g_em = adj.gradient(d_img.float())
    grad = gather(g_mat.cpu().numpy().astype(np.float64), g_em.cpu().numpy().astype(np.float64), check_params,
                  em_mats)

    def loss(mats, rgb):
        set_materials(scene, mats)
        set_emitter_colors(scene, rgb)
        return float(((adj.render().double() - target) ** 2).sum())

    fd = np.zeros(len(check_params))
    for k, p in enumerate(check_params):
        h = eps * max(abs(value_of(start_mats, start_rgb, p)), 1e-2)
        mp, rp = perturb(start_mats, start_rgb, p, h, em_mats)
        mm, rm = perturb(start_mats, start_rgb, p, -h, em_mats)
        fd[k] = (loss(mp, rp) - loss(mm, rm)) / (2.0 * h)
    set_materials(scene, start_mats)
    set_emitter_colors(scene, start_rgb)
    scale = np.maximum(np.abs(fd), 1e-12)
    rel = np.abs(grad - fd) / scale
    return {"adjoint": grad, "fd": fd, "rel_err": rel, "loss": loss(start_mats, start_rgb),
            "frame_max_abs_diff": frame_diff, "frame_max_abs": frame_scale,
            "frame_equal": bool(torch_equal(start_img, frame_img))}


def restir_params(scene_size: float, seed: int = 3, **overrides) -> _abi.Params:
    """Conditional ReSTIR with the large workload's reuse (depth 8, prefix
    length 2, NEE probability 0.3, temporal reuse, 2 suffix spatial rounds of
    5 neighbours, final gather with k = 8 neighbours in a path-length radius)
    and what the adjoint needs: FP32 storage, one final-gather prefix, no
    accumulation."""
    from . import default_params

    kw = dict(renderer_type=_abi.CONDITIONAL_RESTIR, max_path_len=8, nee_prob=0.3, seed=seed, enable_accum=0,
              recon_min_distance=0.01 * scene_size, recon_min_roughness=0.2, prefix_len=2, prefix_enable_temporal=1,
              prefix_enable_spatial=0, suffix_enable_temporal=1, suffix_enable_spatial=1, suffix_spatial_count=5,
              suffix_spatial_rounds=2, gather_n=1, gather_m=9, gather_radius=0.01,
              gather_radius_type=_abi.RADIUS_PATH_LENGTH, window_radius=10, storage=_abi.STORAGE_FP32)
    kw.update(overrides)
    return default_params(scene_size, **kw)


def torch_equal(a, b) -> bool:
    import torch

    return bool(torch.equal(a.double(), b.double()))


def inverse_steps(scene, desc, cams: Sequence[Camera], width: int, height: int, params: _abi.Params,
                  target_mats: np.ndarray, target_rgb: np.ndarray, start_mats: np.ndarray, start_rgb: np.ndarray,
                  steps: int = 10, lr: float = 0.02, estimator: str = "pt", frames: int = 3,
                  free=("diffuse", "roughness", "radiance")) -> dict:
    """Inverse-rendering steps: gradient descent with a backtracking line
    search (steps preconditioned by each parameter's size; the first trial
    moves the steepest parameter by `lr`) on the groups `free` of the parameters the
    adjoints differentiate (every material's diffuse albedo and GGX roughness,
    every emitter's radiance; the other groups stay at the target's values),
    minimising sum of (image - target)^2 over the views.  The
    estimator is frozen at the start parameters -- the path tracer's sampling
    (``PtAdjoint``) or the resampled estimator's prepared frames
    (``RestirAdjoint``, `frames` Conditional ReSTIR frames) -- and the target
    is the same frozen estimator at the target parameters, so the loss is a
    smooth function of the parameters.  Returns the loss before each step and
    after the last, and the parameters' mean absolute relative error to the
    target before and after: over all of them, and over the quarter with the
    largest first gradients (scaled to the parameter), the ones the images
    determine most."""
    em_mats = emitter_materials(desc)
    set_materials(scene, start_mats)
    set_emitter_colors(scene, start_rgb)
    if estimator == "restir":
        adj = RestirAdjoint(scene, width, height, params, len(cams))
        adj.prepare(cams, frames)
        render, grad = adj.render, adj.gradient
    else:
        adj = PtAdjoint(scene, width, height, params)

        def render():
            return adj.render(cams)

        def grad(d):
            return adj.gradient(cams, d)

    set_materials(scene, target_mats)
    set_emitter_colors(scene, target_rgb)
    target = render().double()
    em = np.array([m for m in em_mats], np.int64)
    surf = np.array([m for m in range(len(start_mats)) if m not in set(em_mats)], np.int64)  # not emitters
    ggx = surf[start_mats["roughness"][surf] < 1.0]

    def pack(mats, rgb):
        return np.concatenate([mats["diffuse"][surf].reshape(-1), mats["roughness"][ggx], rgb.reshape(-1)])

    def unpack(x):
        mats, rgb = start_mats.copy(), start_rgb.copy()
        nd, nr = 3 * len(surf), len(ggx)
        mats["diffuse"][surf] = np.clip(x[:nd].reshape(-1, 3), 0.01, 0.99)
        mats["roughness"][ggx] = np.clip(x[nd:nd + nr], 0.02, 1.0)
        rgb = np.maximum(x[nd + nr:].reshape(-1, 3), 0.0).astype(np.float32)
        for e, m in enumerate(em):
            if m >= 0:
                mats["emission"][m] = rgb[e]
        return mats, rgb

    # groups not optimised start (and stay) at the target's values
    sel = np.concatenate([np.full(3 * len(surf), "diffuse" in free), np.full(len(ggx), "roughness" in free),
                          np.full(3 * len(em), "radiance" in free)])
    x_target = pack(target_mats, target_rgb).astype(np.float64)
    x = np.where(sel, pack(start_mats, start_rgb), x_target)
    scale = np.maximum(np.abs(x), 1e-2)  # steps relative to each parameter's size
    losses = []
    rel_err = lambda v: np.abs(v - x_target) / np.maximum(np.abs(x_target), 1e-2)  # noqa: E731
    err0 = rel_err(x)
    observed = None

    def loss_at(v):
        mats, rgb = unpack(v)
        set_materials(scene, mats)
        set_emitter_colors(scene, rgb)
        img = render().double()
        return float(((img - target) ** 2).sum()), img

    cur, img = loss_at(x)
    losses.append(cur)
    alpha = None
    for it in range(steps):
        g_mat, g_em = grad((2.0 * (img - target)).float())
        g_mat = g_mat.double().cpu().numpy()
        g_em = g_em.double().cpu().numpy()
        g_rad = g_em.copy()
        for e, m in enumerate(em):
            if m >= 0:
                g_rad[e] += g_mat[m, 4:7]
        g = np.concatenate([g_mat[surf, 0:3].reshape(-1), g_mat[ggx, 3], g_rad.reshape(-1)]) * scale * sel
        if observed is None:
            observed = sel & (np.abs(g) >= np.quantile(np.abs(g[sel]), 0.75))
        gg = float((g * g).sum())
        if gg == 0.0:
            break
        if alpha is None:
            alpha = lr / float(np.abs(g).max())  # the first trial moves the steepest parameter by lr
        else:
            alpha *= 2.0
        # backtracking (Armijo) along the preconditioned gradient
        for _ in range(20):
            trial = pack(*unpack(x - alpha * scale * g))
            val, timg = loss_at(trial)
            if val <= cur - 1e-4 * alpha * gg:
                break
            alpha *= 0.5
        else:
            break
        x, cur, img = trial, val, timg
        losses.append(cur)
    set_materials(scene, start_mats)
    set_emitter_colors(scene, start_rgb)
    err1 = rel_err(x)
    if observed is None:
        observed = sel
    return {"losses": losses, "param_rel_err_start": float(err0[sel].mean()),
            "param_rel_err_end": float(err1[sel].mean()), "free": list(free), "num_free": int(sel.sum()),
            "observed_rel_err_start": float(err0[observed].mean()), "observed_rel_err_end": float(err1[observed].mean()),
            "num_params": int(len(x)), "num_observed": int(observed.sum()), "estimator": estimator}


def inverse_config_params(desc, num_params: int = 20, seed: int = 3, min_roughness: int = 0) -> List[Param]:
    """`num_params` random parameters of the inverse-rendering config: sphere
    albedos (materials 1..64, 3 channels), GGX roughnesses (odd spheres) and
    emitter radiances; at least `min_roughness` of them roughnesses."""
    rng = np.random.default_rng(seed)
    mats = desc.materials
    em_mats = set(emitter_materials(desc))
    sphere = [m for m in range(1, len(mats)) if m not in em_mats]
    ggx = [m for m in sphere if float(mats["roughness"][m]) < 1.0]
    pool: List[Param] = ([Param("diffuse", m, c) for m in sphere for c in range(3)] +
                         [Param("roughness", m) for m in ggx] +
                         [Param("radiance", e, c) for e in range(len(desc.emitters)) for c in range(3)])
    pick = list(rng.choice(len(pool), size=min(num_params, len(pool)), replace=False))
    have = sum(1 for i in pick if pool[i].kind == "roughness")
    if have < min_roughness:
        first = len(sphere) * 3
        extra = [first + j for j in rng.permutation(len(ggx)) if first + j not in pick][: min_roughness - have]
        drop = [i for i in pick if pool[i].kind != "roughness"][: len(extra)]
        pick = [i for i in pick if i not in drop] + extra
    return [pool[i] for i in pick]


def perturbed_start(desc, seed: int = 3, sigma: float = 0.1):
    """Target (ground-truth) parameters = the scene's; start = target * (1 + N(0,
    sigma)) per parameter (albedos clamped to [0.01, 0.99], roughness to
    [0.02, 1], radiance >= 0)."""
    rng = np.random.default_rng(seed)
    tm = np.array(desc.materials, MATERIAL_DTYPE)
    trgb = np.array([c for c, _, _ in desc.emitters], np.float32).reshape(-1, 3)
    sm, srgb = tm.copy(), trgb.copy()
    em_mats = emitter_materials(desc)
    sm["diffuse"] = np.clip(tm["diffuse"] * (1 + sigma * rng.standard_normal(tm["diffuse"].shape)), 0.01, 0.99)
    ggx = tm["roughness"] < 1.0
    sm["roughness"][ggx] = np.clip(tm["roughness"][ggx] * (1 + sigma * rng.standard_normal(ggx.sum())), 0.02, 1.0)
    srgb = np.maximum(trgb * (1 + sigma * rng.standard_normal(trgb.shape)), 0.0).astype(np.float32)
    for e, m in enumerate(em_mats):
        if m >= 0:
            sm["emission"][m] = srgb[e]
            sm["diffuse"][m] = tm["diffuse"][m]
    return tm, trgb, sm, srgb


def main(argv=None):
    """Central-difference check of the adjoint on the inverse-rendering config:
    the large scene (64 sphere materials, 256 emitters), 8 views of 512 x 512,
    L2 loss against images at the ground-truth parameters, start parameters
    perturbed by N(0, 0.1) relative, 20 random parameters, eps 1e-3, seed 3.
    Prints one JSON line."""
    import argparse
    import json
    import time

    import torch

    from . import Scene, default_params, scenes

    ap = argparse.ArgumentParser()
    ap.add_argument("--views", type=int, default=8)
    ap.add_argument("--res", type=int, default=512)
    ap.add_argument("--params", type=int, default=20)
    ap.add_argument("--eps", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--min-roughness", type=int, default=4, help="at least this many roughness parameters")
    ap.add_argument("--small", action="store_true", help="a 12-sphere room instead of the large scene")
    ap.add_argument("--estimator", default="pt", choices=["pt", "restir"],
                    help="pt: the path tracer; restir: the final gather's resampled estimator")
    ap.add_argument("--frames", type=int, default=3, help="restir: frames rendered before the check")
    ap.add_argument("--inverse-steps", type=int, default=0,
                    help="instead of the check, run this many Adam steps on all parameters and print the losses")
    ap.add_argument("--lr", type=float, default=0.02, help="Adam step, relative to each parameter")
    ap.add_argument("--free", default="diffuse,roughness,radiance",
                    help="inverse steps: the parameter groups optimised (the rest stay at the target)")
    a = ap.parse_args(argv)
    if a.small:
        desc, _ = scenes.sphere_room(num_spheres=12, subdiv=2, num_emitters=12, seed=4)
    else:
        desc, _ = scenes.sphere_room(num_spheres=64, subdiv=5, num_emitters=256, seed=1)
    sc = Scene(desc)
    p = default_params(sc.scene_size, max_path_len=8, nee_prob=0.3, seed=a.seed)
    views = scenes.multiview_cameras([(a.res, a.res)] * a.views, seed=a.seed)
    cams = [c for c, _, _ in views]
    tm, trgb, sm, srgb = perturbed_start(desc, seed=a.seed)
    chk = inverse_config_params(desc, a.params, a.seed, a.min_roughness)
    t0 = time.time()
    if a.inverse_steps:
        q = restir_params(sc.scene_size, a.seed) if a.estimator == "restir" else p
        r = inverse_steps(sc, desc, cams, a.res, a.res, q, tm, trgb, sm, srgb, steps=a.inverse_steps, lr=a.lr,
                          estimator=a.estimator, frames=a.frames, free=tuple(a.free.split(",")))
        torch.cuda.synchronize()
        print(json.dumps({"config": f"inverse rendering: {a.views} views {a.res}x{a.res}, {len(desc.materials)} "
                                    f"materials, {len(desc.emitters)} emitters, Adam lr {a.lr}, seed {a.seed}",
                          **r, "seconds": time.time() - t0}))
        return
    if a.estimator == "restir":
        p = restir_params(sc.scene_size, a.seed)
        r = restir_fd_check(sc, desc, cams, a.res, a.res, p, tm, trgb, sm, srgb, chk, eps=a.eps, frames=a.frames)
    else:
        r = fd_check(sc, desc, cams, a.res, a.res, p, tm, trgb, sm, srgb, chk, eps=a.eps)
    torch.cuda.synchronize()
    big = np.abs(r["fd"]) > 1e-3 * np.abs(r["fd"]).max()
    extra = {k: r[k] for k in ("frame_max_abs_diff", "frame_max_abs", "frame_equal") if k in r}
    print(json.dumps({"config": f"inverse rendering: {a.views} views {a.res}x{a.res}, {len(desc.materials)} materials, "
                                f"{len(desc.emitters)} emitters, {len(chk)} parameters, eps {a.eps}, seed {a.seed}",
                      "estimator": a.estimator, **extra,
                      "max_rel_err": float(r["rel_err"][big].max()) if big.any() else None,
                      "max_rel_err_all": float(r["rel_err"].max()),
                      "params_checked": int(big.sum()), "loss": r["loss"],
                      "params": [f"{q.kind}[{q.index}].{q.channel}" for q in chk],
                      "adjoint": [float(v) for v in r["adjoint"]], "fd": [float(v) for v in r["fd"]],
                      "rel_err": [float(v) for v in r["rel_err"]], "seconds": time.time() - t0}))


if __name__ == "__main__":
    main()
