"""Image quality: relMSE of a rendered frame against a converged reference.

The reference is the unidirectional path tracer of the library
(`TraceCompletePath`, include/graph/restir/path_gen.h:389-472; renderer type
PATH_TRACER) at `spp` samples per pixel, one sample per frame, accumulated in
float64 on the device.  It estimates the same integral as the ReSTIR
estimators, including the reference's NEE convention, so the relMSE measures
resampling error and not a convention mismatch.

relMSE = mean over pixels and channels of (x - ref)^2 / (ref^2 + eps).

On the large workload a single frame's relMSE is dominated by a handful of
fireflies the estimator itself produces (GGX roughness down to 0.05, small
emitters, and an unclamped reconnection Jacobian, include/graph/restir/
path_gen.h:59-72), so the trimmed relMSE -- the same mean without the 0.1% of
pixels with the largest error -- is reported beside it.
"""
from __future__ import annotations

import copy
from typing import Callable, Optional

import numpy as np

from . import _abi
from .scenes import Camera

EPS = 1e-2


def relmse(img: np.ndarray, ref: np.ndarray, eps: float = EPS) -> float:
    img = np.asarray(img, np.float64)
    ref = np.asarray(ref, np.float64)
    if img.shape != ref.shape:
        raise ValueError(f"shape {img.shape} against {ref.shape}")
    return float(np.mean((img - ref) ** 2 / (ref * ref + eps)))


def relmse_trimmed(img: np.ndarray, ref: np.ndarray, drop: float = 1e-3, eps: float = EPS) -> float:
    """relMSE over the pixels whose error is below the (1 - drop) quantile."""
    img = np.asarray(img, np.float64)
    ref = np.asarray(ref, np.float64)
    e = ((img - ref) ** 2 / (ref * ref + eps)).reshape(-1, img.shape[-1]).mean(axis=1)
    keep = np.sort(e)[: max(1, int(round(e.size * (1.0 - drop))))]
    return float(keep.mean())


def reference_image(scene, W: int, H: int, cam: Camera, params, spp: int, stream=None) -> np.ndarray:
    """(H, W, 3) float64 mean of `spp` one-sample path-traced frames."""
    import torch

    from . import Renderer

    p = copy.copy(params)
    p.renderer_type = _abi.PATH_TRACER
    p.enable_accum = 0
    r = Renderer(W, H, scene, p)
    out = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    acc = torch.zeros(W * H * 3, dtype=torch.float64, device="cuda")
    s = stream if stream is not None else torch.cuda.current_stream()
    c = copy.copy(cam)
    c.changed = False
    with torch.cuda.stream(s):
        for _ in range(spp):
            r.launch_frame(c, out.data_ptr(), s.cuda_stream)
            acc += out.double()
    torch.cuda.synchronize()
    r.check_device_errors()
    return (acc / spp).cpu().numpy().reshape(H, W, 3)


def restir_frame(scene, W: int, H: int, cam_of: Callable[[int], Camera], params, frames: int,
                 stream=None) -> np.ndarray:
    """(H, W, 3) float32 image of frame `frames - 1` of a sequence of cameras."""
    import torch

    from . import Renderer

    r = Renderer(W, H, scene, params)
    out = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    s = stream if stream is not None else torch.cuda.current_stream()
    with torch.cuda.stream(s):
        for f in range(frames):
            r.launch_frame(cam_of(f), out.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    r.check_device_errors()
    return out.cpu().numpy().reshape(H, W, 3)


def pt_equal_time(scene, W: int, H: int, cam: Camera, params, ms_budget: float, ref: np.ndarray,
                  seed_offset: int = 7919) -> dict:
    """The plain path tracer at equal time: one-sample frames of `cam` are
    timed here, `equal_time_spp` = ms_budget / ms per sample, and the mean of
    the first floor(equal_time_spp) samples (at least one) and of one sample
    more are scored against `ref`, so a budget near a whole number of samples
    shows both sides.  Its random stream differs from the reference's (seed +
    seed_offset), so the samples are not the reference's own."""
    import torch

    from . import Renderer

    p = copy.copy(params)
    p.renderer_type = _abi.PATH_TRACER
    p.enable_accum = 0
    p.seed = int(p.seed) + seed_offset
    r = Renderer(W, H, scene, p)
    out = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    c = copy.copy(cam)
    c.changed = False
    for _ in range(3):  # warm-up frames (not part of the image)
        r.launch_frame(c, out.data_ptr())
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(5):
        r.launch_frame(c, out.data_ptr())
    t1.record()
    torch.cuda.synchronize()
    ms_spp = t0.elapsed_time(t1) / 5
    lo = max(1, int(ms_budget // ms_spp))
    acc = torch.zeros(W * H * 3, dtype=torch.float64, device="cuda")
    scores = {}
    for n in range(1, lo + 2):
        r.launch_frame(c, out.data_ptr())
        acc += out.double()
        if n >= lo:
            img = (acc / n).cpu().numpy().reshape(H, W, 3)
            scores[str(n)] = {"relmse": relmse(img, ref), "relmse_trimmed_0.1pct": relmse_trimmed(img, ref)}
    r.check_device_errors()
    return {"ms_per_spp": ms_spp, "equal_time_spp": ms_budget / ms_spp, "scores": scores}


def score(scene, W: int, H: int, cam_of: Callable[[int], Camera], params, frames: int, spp: int,
          ref: Optional[np.ndarray] = None) -> dict:
    """relMSE of frame `frames - 1` against the `spp` path-traced reference of
    that frame's camera (computed unless given)."""
    if ref is None:
        ref = reference_image(scene, W, H, cam_of(frames - 1), params, spp)
    img = restir_frame(scene, W, H, cam_of, params, frames)
    return {"relmse": relmse(img, ref), "relmse_trimmed_0.1pct": relmse_trimmed(img, ref), "frame": frames - 1,
            "reference_spp": spp, "eps": EPS,
            "image_mean": float(img.mean()), "reference_mean": float(ref.mean())}
