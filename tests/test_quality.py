"""relMSE scoring: the metric itself on CPU, and on the GPU that Conditional
ReSTIR after 16 frames beats one-sample path tracing against a converged
path-traced reference."""
import numpy as np
import pytest

from crisoptix_b200 import quality, scenes
from helpers import scene_size_of, small_config_params


def test_relmse_definition():
    ref = np.full((2, 2, 3), 2.0)
    img = ref.copy()
    assert quality.relmse(img, ref) == 0.0
    img[0, 0, 0] = 3.0
    assert quality.relmse(img, ref) == pytest.approx(1.0 / (4.0 + quality.EPS) / 12)
    with pytest.raises(ValueError):
        quality.relmse(img[:1], ref)
    # trimming drops the single bad pixel of 1000
    big_ref = np.ones((10, 100, 3))
    big = big_ref.copy()
    big[3, 7] = 50.0
    assert quality.relmse(big, big_ref) > 0.0
    assert quality.relmse_trimmed(big, big_ref) == 0.0


@pytest.mark.gpu
def test_restir_beats_one_sample_path_tracing(cuda_device):
    from crisoptix_b200 import Scene, _abi

    desc, cam = scenes.cornell_box()
    sc = Scene(desc)
    p = small_config_params(scene_size_of(desc))
    W = H = 64
    ref = quality.reference_image(sc, W, H, cam, p, 1024)
    assert np.isfinite(ref).all() and ref.mean() > 0.1
    s = quality.score(sc, W, H, lambda f: cam, p, 16, 1024, ref=ref)
    pt = small_config_params(scene_size_of(desc), renderer_type=_abi.PATH_TRACER)
    one = quality.restir_frame(sc, W, H, lambda f: cam, pt, 1)
    e_pt = quality.relmse(one, ref)
    assert np.isfinite(s["relmse"])
    assert s["relmse"] < e_pt, (s["relmse"], e_pt)


@pytest.mark.gpu
def test_equal_time_path_tracer_scores(cuda_device):
    """The equal-time path tracer arm: whole sample counts either side of the
    budget, each scored, and its samples are not the reference's own (a
    reference made of them would score exactly zero)."""
    from crisoptix_b200 import Scene

    desc, cam = scenes.cornell_box()
    sc = Scene(desc)
    p = small_config_params(scene_size_of(desc))
    W = H = 48
    ref = quality.reference_image(sc, W, H, cam, p, 64)
    r = quality.pt_equal_time(sc, W, H, cam, p, 0.0, ref)
    assert r["ms_per_spp"] > 0.0 and r["equal_time_spp"] == 0.0
    assert sorted(r["scores"]) == ["1", "2"]
    for v in r["scores"].values():
        assert np.isfinite(v["relmse"]) and v["relmse"] > 0.0
    # two samples are closer to the 64-sample reference than one
    assert r["scores"]["2"]["relmse"] < r["scores"]["1"]["relmse"]
