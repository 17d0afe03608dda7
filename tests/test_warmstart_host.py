"""Host-side checks of the learned warm start: the packaged weights, the
standardisation and the network's parameter layout (no GPU)."""

import numpy as np
import torch

from oracle import mlp as om
from sap_warp_b200 import _abi
from sap_warp_b200.warmstart import DEFAULT_WEIGHTS, PARAM_LAYOUT, FeatureNorm, init_params, residual_targets


def test_packaged_weights_are_complete_and_finite():
    z = np.load(DEFAULT_WEIGHTS)
    assert z["params"].shape == (_abi.SAPB_MLP_PARAM_COUNT,)
    assert np.isfinite(z["params"]).all() and np.abs(z["params"]).max() > 0
    for k, size in (("mean", 12), ("inv_std", 12), ("out_scale", 3), ("out_shift", 3)):
        assert z[k].shape == (size,) and np.isfinite(z[k]).all(), k
    assert (z["inv_std"] >= 0).all() and (z["out_scale"] > 0).all()


def test_parameter_layout_matches_the_oracle_and_the_abi():
    assert sum(int(np.prod(s)) for _, s in PARAM_LAYOUT) == _abi.SAPB_MLP_PARAM_COUNT == om.PARAM_COUNT
    assert [k for k, _ in PARAM_LAYOUT] == [k for k in om.offsets()]
    p = init_params(3)
    assert p.dtype == np.float32 and p.shape == (om.PARAM_COUNT,)


def test_feature_norm_encodes_like_the_kernel():
    rng = np.random.default_rng(0)
    raw = rng.normal(size=(100, 12)).astype(np.float32) * 3 + 1
    raw[:, 7] = 0.01  # a constant input gets inv_std 0
    norm = FeatureNorm.from_data(raw, rng.normal(size=(100, 3)))
    assert norm.inv_std[7] == 0
    x = norm.encode(torch.from_numpy(raw))
    assert x.dtype == torch.int16 and x.shape == (100, 16)
    want = om.bf16_bits((raw - norm.mean) * norm.inv_std).view(np.int16)
    np.testing.assert_array_equal(x[:, :12].numpy(), want)
    assert (x[:, 12:] == 0).all()


def test_residual_targets_subtract_previous_impulses_and_clip():
    raw = torch.zeros(1000, 12)
    raw[:, 9:12] = 1.0
    u = torch.randn(1000, 3)
    u[0] = 1e6
    r = residual_targets(raw, u, clip_quantile=0.01)
    assert r.shape == (1000, 3) and float(r.max()) < 1e3
    r0 = residual_targets(raw, u, clip_quantile=0.0)
    torch.testing.assert_close(r0, u - 1.0)
