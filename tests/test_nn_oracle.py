"""The CPU oracle of the warm-start network: its analytic gradients against central finite
differences (unquantised, float64), and the bf16 rounding helper against torch's."""
import numpy as np

from oracle import nn_oracle as no


def _params(rng):
    return no.flatten([(rng.standard_normal((co, 3, 3, ci)) * np.sqrt(2 / (9 * ci)), 0.1 * rng.standard_normal(co))
                       for ci, co, _, _ in no.LAYERS])


def test_param_count():
    assert no.param_count() == 212432


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    x = rng.standard_normal((2, 8, 16, 16))
    x[..., 3:] = 0
    t = rng.standard_normal((2, 8, 16))
    _, g = no.net_loss_grad(p, x, t, quant=False)
    # one parameter from every layer's weights and biases, plus random ones
    idx = []
    o = 0
    for ci, co, _, _ in no.LAYERS:
        idx += [o + (7 * ci) % (co * 9 * ci), o + co * 9 * ci]
        o += co * 9 * ci + co
    idx += list(rng.choice(p.size, 8, replace=False))
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (no.net_loss_grad(pp, x, t, False)[0] - no.net_loss_grad(pm, x, t, False)[0]) / (2 * h)
        assert abs(g[i] - fd) <= 1e-6 * abs(fd) + 1e-9, (i, g[i], fd)


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.standard_normal(1000) * 10.0 ** rng.integers(-20, 20, 1000),
                        [0.0, -0.0, 1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -9, 65504.0]]).astype(np.float32)
    ref = torch.tensor(x).to(torch.bfloat16).float().numpy().astype(np.float64)
    assert np.array_equal(no.bf16(x), ref)
