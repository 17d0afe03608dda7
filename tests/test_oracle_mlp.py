"""The numpy network oracle (oracle/mlp.py) against torch float64 autograd and
torch's BF16 rounding, on the CPU."""

import numpy as np
import torch

from oracle import mlp as om


def torch_net(params: np.ndarray, x: np.ndarray):
    """float64 autograd of the unrounded network with BF16-rounded weights."""
    p = om.unpack(params)
    leaves = {}
    for k, v in p.items():
        a = om.bf16(v) if k.startswith("W") else v
        leaves[k] = torch.tensor(a.astype(np.float64), requires_grad=True)
    xt = torch.tensor(np.asarray(x, np.float64)[:, :om.IN])

    def gelu(z):
        return 0.5 * z * (1.0 + torch.tanh(om.GELU_C * (z + om.GELU_A * z ** 3)))

    h = gelu(xt @ leaves["W1"].T + leaves["b1"])
    h = gelu(h @ leaves["W2"].T + leaves["b2"])
    h = gelu(h @ leaves["W3"].T + leaves["b3"])
    y = h @ leaves["W4"].T + leaves["b4"]
    return y, leaves


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=4096).astype(np.float32) * 10.0 ** rng.integers(-8, 8, 4096),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e38], np.float32)])
    ref = torch.tensor(x).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(om.bf16(x), ref)
    np.testing.assert_array_equal(om.from_bf16_bits(om.bf16_bits(x)), ref)


def test_backward_matches_float64_autograd():
    rng = np.random.default_rng(1)
    params = om.init_params(3)
    params[om.offsets()["W4"][0]:] *= 10.0  # a non-trivial output layer
    x = rng.normal(size=(64, om.IN)).astype(np.float32)
    t = rng.normal(size=(64, 3))
    loss, grad, f = om.backward(params, x, t, mirror=False)
    y, leaves = torch_net(params, x)
    tl = ((y - torch.tensor(t)) ** 2).mean()
    tl.backward()
    np.testing.assert_allclose(f["y"], y.detach().numpy(), rtol=1e-12, atol=1e-12)
    assert abs(loss / (3 * 64) - tl.item()) <= 1e-12 * max(1.0, tl.item())
    g = om.unpack(grad)
    for k, leaf in leaves.items():
        np.testing.assert_allclose(g[k], leaf.grad.numpy(), rtol=1e-5, atol=1e-9, err_msg=k)


def test_mirrored_rounding_stays_close_to_exact():
    rng = np.random.default_rng(2)
    params = om.init_params(4)
    x = om.bf16(rng.normal(size=(256, om.IN)))
    t = rng.normal(size=(256, 3))
    _, g_m, f_m = om.backward(params, x, t, mirror=True)
    _, g_x, f_x = om.backward(params, x, t, mirror=False)
    assert np.abs(f_m["y"] - f_x["y"]).max() <= 2e-2 * np.abs(f_x["y"]).max()
    gm, gx = om.unpack(g_m), om.unpack(g_x)
    for k in gx:
        err = np.linalg.norm(gm[k] - gx[k]) / max(np.linalg.norm(gx[k]), 1e-30)
        assert err < 5e-2, (k, err)


def test_adam_step_decreases_quadratic():
    p = np.ones(om.PARAM_COUNT, np.float32)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    for step in range(1, 50):
        g = 2.0 * p
        p, m, v = om.adam(p, g, m, v, step, lr=0.05)
    assert np.all(np.abs(p) < 0.5)
