"""Path-replay adjoint of the final gather's resampled estimator
(crisb_restir_adjoint_*): the frozen estimator reproduces the frame it
replays, its gradients of an L2 image loss match central differences of the
same frozen estimator (float64 sums), the torch.autograd.Function wrapper
matches the direct call, and unsupported configurations are rejected."""
import numpy as np
import pytest
import torch

from crisoptix_b200 import Renderer, Scene, _abi, adjoint, scenes
from helpers import large_config_params, scene_size_of

pytestmark = pytest.mark.gpu


def _room():
    return scenes.sphere_room(num_spheres=12, subdiv=2, num_emitters=12, seed=4)


def _params(desc, **kw):
    base = dict(max_path_len=6, enable_accum=0, gather_n=1, storage=_abi.STORAGE_FP32)
    base.update(kw)
    return large_config_params(scene_size_of(desc), **base)


def test_frozen_estimator_reproduces_the_frame(cuda_device):
    """At the tables the frame was rendered with, the re-traced estimator gives
    the frame's own gather values bit for bit (neighbour terms re-trace each
    neighbour sample's path past its reconnection vertex from its seed)."""
    desc, cam = _room()
    sc = Scene(desc)
    adj = adjoint.RestirAdjoint(sc, 96, 64, _params(desc), 2)
    cams = [cam, scenes.orbit_camera(cam, 15, 60)]
    frame = adj.prepare(cams, frames=3)
    img = adj.render()
    assert float(frame.abs().sum()) > 0
    np.testing.assert_array_equal(img.cpu().numpy(), frame.cpu().numpy())


def test_restir_adjoint_matches_central_differences(cuda_device):
    desc, cam = _room()
    sc = Scene(desc)
    tm, trgb, sm, srgb = adjoint.perturbed_start(desc, seed=3)
    params = adjoint.inverse_config_params(desc, num_params=20, seed=3, min_roughness=5)
    cams = [cam, scenes.orbit_camera(cam, 15, 60)]
    r = adjoint.restir_fd_check(sc, desc, cams, 96, 64, _params(desc), tm, trgb, sm, srgb, params, eps=1e-3,
                                frames=3)
    big = np.abs(r["fd"]) > 1e-3 * np.abs(r["fd"]).max()
    assert big.sum() >= 10, r
    assert r["rel_err"][big].max() < 1e-2, (r["rel_err"], r["adjoint"], r["fd"])


def test_restir_autograd_function_matches_direct_call(cuda_device):
    desc, cam = _room()
    sc = Scene(desc)
    base = adjoint.get_materials(sc)
    adj = adjoint.RestirAdjoint(sc, 40, 32, _params(desc), 1)
    adj.prepare([cam], frames=2)
    RestirImage = adjoint.restir_image_function()
    diffuse = torch.tensor(base["diffuse"], dtype=torch.float64, requires_grad=True)
    rough = torch.tensor(base["roughness"], dtype=torch.float64, requires_grad=True)
    emission = torch.tensor(base["emission"], dtype=torch.float64, requires_grad=True)
    rgb = torch.tensor(np.array([c for c, _, _ in desc.emitters]), dtype=torch.float64, requires_grad=True)
    img = RestirImage.apply(diffuse, rough, emission, rgb, adj, base)
    loss = (img.double() ** 2).sum()
    loss.backward()
    g_mat, g_em = adj.gradient(2.0 * img.detach())
    np.testing.assert_allclose(diffuse.grad.numpy(), g_mat[:, 0:3].cpu().numpy(), rtol=1e-6)
    np.testing.assert_allclose(rgb.grad.numpy(), g_em.cpu().numpy(), rtol=1e-6)
    assert np.abs(rgb.grad.numpy()).sum() > 0 and np.abs(diffuse.grad.numpy()).sum() > 0


def test_restir_adjoint_rejects_unsupported_configurations(cuda_device):
    desc, cam = _room()
    sc = Scene(desc)
    out = torch.zeros(32 * 24 * 3, device="cuda")
    g_mat = torch.zeros(len(desc.materials) * 7, device="cuda")
    g_em = torch.zeros(len(desc.emitters) * 3, device="cuda")
    # not enabled before the frame
    r = Renderer(32, 24, sc, _params(desc))
    r.launch_frame(cam, out.data_ptr())
    with pytest.raises(RuntimeError):
        r.restir_adjoint_forward(out.data_ptr())
    r.restir_adjoint_enable(True)
    with pytest.raises(RuntimeError):  # the last frame was rendered before enabling
        r.restir_adjoint_backward(out.data_ptr(), g_mat.data_ptr(), g_em.data_ptr())
    r.launch_frame(cam, out.data_ptr())
    r.restir_adjoint_forward(out.data_ptr())
    r.set_job_capacity(4)  # reallocates the frame's shift results: its adjoint ends
    with pytest.raises(RuntimeError):
        r.restir_adjoint_forward(out.data_ptr())
    r.launch_frame(cam, out.data_ptr())
    r.restir_adjoint_forward(out.data_ptr())
    for kw in (dict(storage=_abi.STORAGE_FP16), dict(gather_n=2), dict(renderer_type=_abi.PATH_TRACER)):
        r = Renderer(32, 24, sc, _params(desc, **kw))
        r.restir_adjoint_enable(True)
        r.launch_frame(cam, out.data_ptr())
        with pytest.raises(RuntimeError):
            r.restir_adjoint_forward(out.data_ptr())
    torch.cuda.synchronize()


def test_restir_adjoint_at_the_inverse_rendering_config(cuda_device):
    """The inverse-rendering config at its stated size (the large scene's 992
    parameters, 8 views of 512 x 512, 20 parameters drawn with seed 3, start
    perturbed by N(0, 0.1) relative, eps 1e-3, float64 loss sums), on the
    resampled estimator after 3 Conditional ReSTIR frames per view."""
    desc, _ = scenes.sphere_room(num_spheres=64, subdiv=5, num_emitters=256, seed=1)
    sc = Scene(desc)
    assert sc.num_triangles == 1310988
    p = adjoint.restir_params(sc.scene_size, seed=3)
    cams = [c for c, _, _ in scenes.multiview_cameras([(512, 512)] * 8, seed=3)]
    tm, trgb, sm, srgb = adjoint.perturbed_start(desc, seed=3)
    params = adjoint.inverse_config_params(desc, 20, 3)
    r = adjoint.restir_fd_check(sc, desc, cams, 512, 512, p, tm, trgb, sm, srgb, params, eps=1e-3, frames=3)
    # the gradients span seven decades here (fireflies of the reference's
    # unclamped reconnection Jacobian weigh on the loss): every parameter above
    # 1e-6 of the largest is checked
    big = np.abs(r["fd"]) > 1e-6 * np.abs(r["fd"]).max()
    assert big.sum() >= 15, r
    assert r["rel_err"][big].max() < 1e-2, (r["rel_err"], r["adjoint"], r["fd"])
    assert r["frame_equal"], r


def _grad_samples(grad_fn, frames):
    """Mean and standard error over `frames` of the per-material diffuse and
    roughness gradients grad_fn(frame) returns."""
    g = []
    for f in range(frames):
        g_mat, g_em = grad_fn(f)
        g.append(g_mat.double().cpu().numpy()[:, 0:4].reshape(-1))
    g = np.array(g)
    return g.mean(0), g.std(0) / np.sqrt(frames)


def test_canonical_gradient_matches_the_path_tracer_gradient(cuda_device):
    """Against the gradient of the plain unidirectional estimator.  Without
    neighbours (gather_m 1) the final gather is the canonical prefix + suffix
    path: vertices 1..7 of a depth-8 configuration with prefix length 2, NEE
    forced at vertex 7 -- in expectation the path tracer of depth 7, apart
    from the primary-hit emission term.  The mean gradients of loss = sum of
    the image over 256 frames (diffuse albedo and roughness of every
    material) agree with the path-tracer adjoint's within their standard
    errors."""
    desc, cam = scenes.cornell_box()
    sc = Scene(desc)
    W = H = 128
    frames = 256
    ones = torch.ones(1, H, W, 3, device="cuda")
    pt = adjoint.PtAdjoint(sc, W, H, adjoint.restir_params(sc.scene_size, seed=3, renderer_type=_abi.PATH_TRACER,
                                                          max_path_len=7))
    mp, sp = _grad_samples(lambda f: pt.gradient([cam], ones, frame=f), frames)
    ra = adjoint.RestirAdjoint(sc, W, H, adjoint.restir_params(sc.scene_size, seed=3, gather_m=1), 1)
    ra.prepare([cam], frames=1)

    def restir_grad(f):
        ra.prepare([cam], frames=1)
        return ra.gradient(ones)

    mr, sr = _grad_samples(restir_grad, frames)
    top = np.argsort(-np.abs(mp))[:12]
    z = (mr[top] - mp[top]) / np.sqrt(sp[top] ** 2 + sr[top] ** 2)
    assert np.abs(z).max() < 4.0, (z, mp[top], mr[top], sp[top], sr[top])
    # where the standard errors are small the means agree within a few per cent
    tight = np.sqrt(sp[top] ** 2 + sr[top] ** 2) < 0.02 * np.abs(mp[top])
    assert tight.sum() >= 6, (mp[top], sp[top], sr[top])
    assert np.all(np.abs(mr[top][tight] / mp[top][tight] - 1.0) < 0.08), (mp[top], mr[top])


@pytest.mark.parametrize("estimator", ["pt", "restir"])
def test_inverse_rendering_steps_reduce_the_loss(cuda_device, estimator):
    """Adam on every diffuse albedo of the 12-sphere room (start perturbed by
    N(0, 0.1) relative; roughness and radiance at the target, which removes
    the albedo-radiance scale ambiguity), each step one adjoint backward
    pass: the loss against the target images falls, and the albedos the
    images determine (the quarter with the largest first gradients) move
    toward the target."""
    desc, cam = _room()
    sc = Scene(desc)
    tm, trgb, sm, srgb = adjoint.perturbed_start(desc, seed=3)
    cams = [cam, scenes.orbit_camera(cam, 15, 60)]
    p = _params(desc) if estimator == "restir" else large_config_params(scene_size_of(desc), max_path_len=6)
    r = adjoint.inverse_steps(sc, desc, cams, 96, 64, p, tm, trgb, sm, srgb, steps=15, lr=0.02,
                              estimator=estimator, free=("diffuse",))
    assert r["losses"][-1] < 0.5 * r["losses"][0], r
    assert r["observed_rel_err_end"] < r["observed_rel_err_start"], r
