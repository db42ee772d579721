"""Path-replay adjoint: gradients of an L2 image loss against central
differences of the same frozen-sampling estimator (float64 sums), and the
torch.autograd.Function wrapper against the direct call."""
import numpy as np
import pytest
import torch

from crisoptix_b200 import Scene, adjoint, scenes
from helpers import large_config_params, scene_size_of


def _room():
    desc, cam = scenes.sphere_room(num_spheres=12, subdiv=2, num_emitters=12, seed=4)
    return desc, cam


@pytest.mark.gpu
def test_adjoint_matches_central_differences(cuda_device):
    desc, cam = _room()
    sc = Scene(desc)
    p = large_config_params(scene_size_of(desc), max_path_len=6)
    tm, trgb, sm, srgb = adjoint.perturbed_start(desc, seed=3)
    params = adjoint.inverse_config_params(desc, num_params=20, seed=3, min_roughness=5)
    assert sum(q.kind == "roughness" for q in params) >= 5
    cams = [cam, scenes.orbit_camera(cam, 15, 60)]
    r = adjoint.fd_check(sc, desc, cams, 96, 64, p, tm, trgb, sm, srgb, params, eps=1e-3)
    big = np.abs(r["fd"]) > 1e-3 * np.abs(r["fd"]).max()
    assert big.sum() >= 10, r
    assert r["rel_err"][big].max() < 1e-2, (r["rel_err"], r["adjoint"], r["fd"])


@pytest.mark.gpu
def test_frozen_estimator_equals_path_tracer_at_frozen_parameters(cuda_device):
    from crisoptix_b200 import Renderer, _abi

    desc, cam = _room()
    sc = Scene(desc)
    p = large_config_params(scene_size_of(desc), max_path_len=6, renderer_type=_abi.PATH_TRACER)
    adj = adjoint.PtAdjoint(sc, 48, 32, p)
    img = adj.render([cam], 0)[0].reshape(-1)
    r = Renderer(48, 32, sc, p)
    out = torch.zeros(48 * 32 * 3, device="cuda")
    r.launch_frame(cam, out.data_ptr())  # frame counter 0: the same seeds
    torch.cuda.synchronize()
    np.testing.assert_allclose(img.cpu().numpy(), out.cpu().numpy(), rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_autograd_function_matches_direct_call(cuda_device):
    desc, cam = _room()
    sc = Scene(desc)
    p = large_config_params(scene_size_of(desc), max_path_len=6)
    base = adjoint.get_materials(sc)
    adj = adjoint.PtAdjoint(sc, 40, 32, p)
    PtImage = adjoint.pt_image_function()
    diffuse = torch.tensor(base["diffuse"], dtype=torch.float64, requires_grad=True)
    rough = torch.tensor(base["roughness"], dtype=torch.float64, requires_grad=True)
    emission = torch.tensor(base["emission"], dtype=torch.float64, requires_grad=True)
    rgb = torch.tensor(np.array([c for c, _, _ in desc.emitters]), dtype=torch.float64, requires_grad=True)
    img = PtImage.apply(diffuse, rough, emission, rgb, adj, base, [cam], 0)
    loss = (img.double() ** 2).sum()
    loss.backward()
    g_mat, g_em = adj.gradient([cam], 2.0 * img.detach(), 0)
    np.testing.assert_allclose(diffuse.grad.numpy(), g_mat[:, 0:3].cpu().numpy(), rtol=1e-6)
    np.testing.assert_allclose(rgb.grad.numpy(), g_em.cpu().numpy(), rtol=1e-6)
    assert np.abs(rgb.grad.numpy()).sum() > 0 and np.abs(diffuse.grad.numpy()).sum() > 0


@pytest.mark.gpu
def test_adjoint_at_the_inverse_rendering_config(cuda_device):
    """The inverse-rendering config at its stated size: the large scene
    (1,310,988 triangles; its 64 sphere materials give 64 x 3 albedos and 32
    GGX roughnesses, its 256 emitters 256 x 3 radiances -- 992 parameters), 8
    views of 512 x 512, L2 loss against images at the ground-truth
    parameters, start perturbed by N(0, 0.1) relative, 20 parameters drawn
    with seed 3, central differences with eps 1e-3 summed in float64."""
    from crisoptix_b200 import default_params

    desc, _ = scenes.sphere_room(num_spheres=64, subdiv=5, num_emitters=256, seed=1)
    sc = Scene(desc)
    assert sc.num_triangles == 1310988
    p = default_params(sc.scene_size, max_path_len=8, nee_prob=0.3, seed=3)
    cams = [c for c, _, _ in scenes.multiview_cameras([(512, 512)] * 8, seed=3)]
    tm, trgb, sm, srgb = adjoint.perturbed_start(desc, seed=3)
    params = adjoint.inverse_config_params(desc, 20, 3)
    pool = 64 * 3 + int((tm["roughness"][1:65] < 1.0).sum()) + 256 * 3
    assert pool == 992
    r = adjoint.fd_check(sc, desc, cams, 512, 512, p, tm, trgb, sm, srgb, params, eps=1e-3)
    big = np.abs(r["fd"]) > 1e-3 * np.abs(r["fd"]).max()
    assert big.sum() >= 10, r
    assert r["rel_err"][big].max() < 1e-2, (r["rel_err"], r["adjoint"], r["fd"])
