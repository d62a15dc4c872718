"""Inverse rendering through the adjoint: Adam lowers the image loss and recovers g."""
import pytest
import torch

from helpers import sb
from spectral_b200 import configs, inverse

pytestmark = pytest.mark.gpu


def test_adam_reduces_image_loss_and_parameter_error():
    s, c, ex = configs.volume_scene(width=48, height=48, medium_slices=16, medium_stacks=17, depth=8)
    c.kernel = "mega"
    with sb.Renderer(s, c, eems=ex["eems"], cmf=ex["cmf"]) as r:
        hidden = inverse.Params.from_scene_params(inverse.scene_params(7), "cuda")
        init = inverse.Params.from_scene_params(inverse.scene_params(7), "cuda")
        # perturb the absorption spectrum and g away from the hidden values
        init.sigma_a = init.sigma_a * 2.0
        init.g = torch.as_tensor(0.2, dtype=torch.float64, device="cuda")
        assert hidden.count() == 79
        target = inverse.render_target(r, hidden, blocks=40)
        fit, hist = inverse.run(r, target, init, iterations=40, lr=5e-2, blocks=2)
        e0 = inverse.parameter_error(init, hidden)
        e1 = inverse.parameter_error(fit, hidden)
        assert all(torch.isfinite(torch.tensor(hist)))
        assert sum(hist[-5:]) < 0.5 * sum(hist[:5]), hist
        # g is identifiable from the XYZ image; 25-band spectra are not (metamerism)
        assert e1["g"] < 0.5 * e0["g"], (e0, e1)
        assert r.check_device() == 0
