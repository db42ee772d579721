"""Golden vectors (tests/golden/*.npz, made by tests/golden/make_golden.py):
the oracle on CPU, and the CUDA path on the GPU, must reproduce them bit for
bit."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402

from crisoptix_b200 import _abi  # noqa: E402


def load(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


@pytest.mark.parametrize("name", list(mg.CASES))
def test_oracle_reproduces_golden(name):
    g = load(name)
    img, state = mg.run_oracle(mg.CASES[name])
    assert img.tobytes() == g["image"].tobytes()
    for k, v in state.items():
        assert v.view(np.uint8).tobytes() == g["buf" + k].tobytes(), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(mg.CASES))
def test_cuda_path_reproduces_golden(cuda_device, name):
    import torch

    from crisoptix_b200 import Renderer, Scene, scenes

    case = mg.CASES[name]
    desc, cam, p, cam_fn = mg.case_inputs(case)
    g = load(name)
    # the fixtures were made from the scene's float64 flattening: give the
    # GPU exactly that triangle soup
    r = Renderer(case["W"], case["H"], Scene(scenes.flat_scene(desc)), p)
    out = torch.zeros(case["W"] * case["H"] * 3, dtype=torch.float32, device="cuda")
    for f in range(case["frames"]):
        r.launch_frame(cam_fn(cam, f), out.data_ptr())
    torch.cuda.synchronize()
    r.check_device_errors()
    assert out.cpu().numpy().tobytes() == g["image"].tobytes()
    for k in mg.STATE:
        assert r.debug_read(k).view(np.uint8).tobytes() == g["buf" + str(k)].tobytes(), k
