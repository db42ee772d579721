"""Host logic of the adjoints (no GPU): the inverse-rendering parameter pool,
the perturbed start, and how gradients and perturbations map onto the
material and emitter tables (a radiance is the emitter's colour and its
material's emission at once)."""
import numpy as np

from crisoptix_b200 import adjoint, scenes


def _large():
    desc, _ = scenes.sphere_room(num_spheres=64, subdiv=5, num_emitters=256, seed=1)
    return desc


def test_inverse_config_pool_and_draw():
    """64 sphere albedos x 3, the GGX spheres' roughness and 256 radiances x 3:
    992 parameters; 20 drawn with seed 3, reproducibly, without repeats."""
    desc = _large()
    em = adjoint.emitter_materials(desc)
    assert len(em) == 256 and all(m >= 0 for m in em)
    mats = desc.materials
    spheres = [m for m in range(1, len(mats)) if m not in set(em)]
    assert len(spheres) == 64
    ggx = [m for m in spheres if float(mats["roughness"][m]) < 1.0]
    assert 64 * 3 + len(ggx) + 256 * 3 == 992
    a = adjoint.inverse_config_params(desc, 20, 3)
    b = adjoint.inverse_config_params(desc, 20, 3)
    key = [(p.kind, p.index, p.channel) for p in a]
    assert key == [(p.kind, p.index, p.channel) for p in b]
    assert len(set(key)) == 20
    forced = adjoint.inverse_config_params(desc, 20, 3, min_roughness=5)
    assert sum(p.kind == "roughness" for p in forced) >= 5 and len(forced) == 20


def test_perturbed_start_keeps_ranges_and_ties_radiance_to_emission():
    desc = _large()
    tm, trgb, sm, srgb = adjoint.perturbed_start(desc, seed=3, sigma=0.1)
    assert np.all((sm["diffuse"] >= 0.01) & (sm["diffuse"] <= 0.99))
    ggx = tm["roughness"] < 1.0
    assert np.all((sm["roughness"][ggx] >= 0.02) & (sm["roughness"][ggx] <= 1.0))
    assert np.all(sm["roughness"][~ggx] == tm["roughness"][~ggx])
    assert np.all(srgb >= 0.0)
    for e, m in enumerate(adjoint.emitter_materials(desc)):
        np.testing.assert_array_equal(sm["emission"][m], srgb[e])
        np.testing.assert_array_equal(sm["diffuse"][m], tm["diffuse"][m])
    rel = np.abs(sm["diffuse"][1:65] / tm["diffuse"][1:65] - 1.0)
    assert 0.02 < float(np.median(rel)) < 0.2  # N(0, 0.1) relative


def test_gather_and_perturb_agree_on_radiance():
    """gather() adds the emitter-colour and emission gradients of a radiance;
    perturb() moves both the colour and the emission by the same step."""
    desc, _ = scenes.sphere_room(num_spheres=12, subdiv=2, num_emitters=12, seed=4)
    em = adjoint.emitter_materials(desc)
    nm, ne = len(desc.materials), len(desc.emitters)
    g_mat = np.arange(nm * 7, dtype=np.float64).reshape(nm, 7)
    g_em = -np.arange(ne * 3, dtype=np.float64).reshape(ne, 3)
    ps = [adjoint.Param("diffuse", 3, 1), adjoint.Param("roughness", 2), adjoint.Param("radiance", 5, 2)]
    g = adjoint.gather(g_mat, g_em, ps, em)
    assert g[0] == g_mat[3, 1] and g[1] == g_mat[2, 3]
    assert g[2] == g_em[5, 2] + g_mat[em[5], 6]
    mats = np.array(desc.materials)
    rgb = np.array([c for c, _, _ in desc.emitters], np.float32).reshape(-1, 3)
    m2, r2 = adjoint.perturb(mats, rgb, ps[2], 0.25, em)
    assert np.isclose(r2[5, 2] - rgb[5, 2], 0.25)
    assert np.isclose(m2["emission"][em[5], 2] - mats["emission"][em[5], 2], 0.25)
    assert np.array_equal(m2["diffuse"], mats["diffuse"]) and np.array_equal(np.delete(r2, 5, 0), np.delete(rgb, 5, 0))
    assert adjoint.value_of(mats, rgb, ps[0]) == float(mats["diffuse"][3, 1])


def test_restir_params_meet_the_adjoint_requirements():
    from crisoptix_b200 import _abi

    p = adjoint.restir_params(10.0, seed=3)
    assert p.renderer_type == _abi.CONDITIONAL_RESTIR and p.gather_n == 1 and p.enable_accum == 0
    assert p.storage == _abi.STORAGE_FP32 and p.gather_m == 9 and p.max_path_len <= 16
    q = adjoint.restir_params(10.0, seed=3, gather_m=1)
    assert q.gather_m == 1 and q.seed == 3
