"""Known-answer and consistency tests that pin the CPU oracle's projection.

The reference ships no golden vectors, so the oracle is pinned here against
closed-form answers of the reference's own formulas
(sim/contact_solve.py:743-921) and against calculus identities they must
satisfy (d cost / d vc = -gamma, G = -d gamma / d vc).
"""

import json
from pathlib import Path

import numpy as np
import pytest

from tests import sap_numpy as sn

GOLDEN = Path(__file__).resolve().parent / "golden" / "known_answers.json"


def _consts(phi0=-1e-3, w=0.5, mu=0.6, k=1e5, tau=0.01, dt=2e-3):
    rt, rn, vhat = sn.contact_constants(np.array(phi0), np.array(w), np.array(mu), np.array(k), np.array(tau), dt=dt)
    return float(rt), float(rn), float(vhat)


def test_known_answers_file(oracle):
    """Every golden case (closed-form, see tests/golden/make_known_answers.py)."""
    cases = json.loads(GOLDEN.read_text())["projection"]
    assert len(cases) >= 8
    for case in cases:
        got = oracle.project(case["vc"], case["phi0"], case["w"], case["mu"], case["k"], case["tau"],
                             dt=case["dt"])
        assert got["mode"] == case["mode"], case["name"]
        np.testing.assert_allclose(got["gamma"], case["gamma"], rtol=1e-12, atol=1e-14, err_msg=case["name"])
        np.testing.assert_allclose(got["cost"], case["cost"], rtol=1e-12, atol=1e-18, err_msg=case["name"])
        np.testing.assert_allclose(got["G"], np.array(case["G"]), rtol=1e-10, atol=1e-8, err_msg=case["name"])


def test_stiction_regime(oracle):
    rt, rn, vhat = _consts()
    vc = [1e-6, -2e-6, 0.0]
    got = oracle.project(vc, -1e-3, 0.5, 0.6, 1e5, 0.01)
    y = np.array([-vc[0] / rt, -vc[1] / rt, (vhat - vc[2]) / rn])
    assert np.hypot(y[0], y[1]) <= 0.6 * y[2]
    assert got["mode"] == 1
    np.testing.assert_allclose(got["gamma"], y, rtol=1e-13)
    np.testing.assert_allclose(got["G"], np.diag([1 / rt, 1 / rt, 1 / rn]), rtol=1e-13)


def test_sliding_regime(oracle):
    rt, rn, vhat = _consts()
    vc = [0.3, 0.1, 0.0]
    got = oracle.project(vc, -1e-3, 0.5, 0.6, 1e5, 0.01)
    y = np.array([-vc[0] / rt, -vc[1] / rt, (vhat - vc[2]) / rn])
    yr = np.sqrt(y[0] ** 2 + y[1] ** 2 + 1e-14)
    mu_hat = 0.6 * rt / rn
    mu_tilde2 = 0.36 * rt / rn
    gn = (y[2] + mu_hat * yr) / (1 + mu_tilde2)
    assert got["mode"] == 2
    np.testing.assert_allclose(got["gamma"], [0.6 * gn * y[0] / yr, 0.6 * gn * y[1] / yr, gn], rtol=1e-12)


def test_separation_and_frictionless(oracle):
    got = oracle.project([0.0, 0.0, 1.0], 1e-3, 0.5, 0.6, 1e5, 0.01)  # separating
    assert got["mode"] == 0 and np.all(got["gamma"] == 0) and got["cost"] == 0
    rt, rn, vhat = _consts(mu=0.0)
    got = oracle.project([0.2, 0.0, -0.01], -1e-3, 0.5, 0.0, 1e5, 0.01)
    assert got["mode"] == 3
    np.testing.assert_allclose(got["gamma"], [0, 0, (vhat + 0.01) / rn], rtol=1e-13)


@pytest.mark.parametrize("seed", range(6))
def test_gradient_and_hessian_identities(oracle, seed):
    """d cost / d vc = -gamma and G = -d gamma / d vc (central differences)."""
    rng = np.random.default_rng(seed)
    for _ in range(40):
        vc = rng.normal(scale=[0.05, 0.05, 0.02])
        phi0 = rng.uniform(-2e-3, 0)
        w, mu = rng.uniform(0.05, 2.0), rng.uniform(0.1, 1.0)
        k, tau = 10 ** rng.uniform(4, 8), rng.uniform(0, 0.02)
        base = oracle.project(vc, phi0, w, mu, k, tau)
        h = 1e-7 * max(1e-3, np.abs(vc).max())
        grad = np.zeros(3)
        jac = np.zeros((3, 3))
        modes = set()
        for j in range(3):
            e = np.zeros(3)
            e[j] = h
            p = oracle.project(vc + e, phi0, w, mu, k, tau)
            m = oracle.project(vc - e, phi0, w, mu, k, tau)
            modes |= {p["mode"], m["mode"]}
            grad[j] = (p["cost"] - m["cost"]) / (2 * h)
            jac[:, j] = -(p["gamma"] - m["gamma"]) / (2 * h)
        if modes != {base["mode"]}:
            continue  # straddles a regime boundary
        scale = max(1.0, np.abs(base["gamma"]).max())
        np.testing.assert_allclose(grad, -base["gamma"], rtol=1e-5, atol=1e-6 * scale)
        gscale = max(1.0, np.abs(base["G"]).max())
        np.testing.assert_allclose(jac, base["G"], rtol=1e-4, atol=1e-5 * gscale)
        # G is symmetric positive semi-definite
        np.testing.assert_allclose(base["G"], base["G"].T, rtol=1e-10, atol=1e-12 * gscale)
        assert np.linalg.eigvalsh(0.5 * (base["G"] + base["G"].T)).min() > -1e-9 * gscale


def test_projection_matches_numpy_statement(oracle):
    rng = np.random.default_rng(7)
    for _ in range(200):
        vc = rng.normal(scale=0.05, size=3)
        phi0, w, mu = rng.uniform(-2e-3, 1e-3), rng.uniform(0.05, 2.0), rng.uniform(0.0, 1.0)
        k, tau = 10 ** rng.uniform(4, 10), rng.uniform(0, 0.02)
        got = oracle.project(vc, phi0, w, mu, k, tau)
        rt, rn, vhat = sn.contact_constants(*map(np.array, (phi0, w, mu, k, tau)))
        gamma, mode = sn.project(vc[None], np.array([mu]), rt, rn, vhat)
        assert got["mode"] == int(mode[0])
        np.testing.assert_allclose(got["gamma"], gamma[0], rtol=1e-12, atol=1e-300)


def test_pd_gains_and_clamp(oracle):
    lib = oracle.load()
    import ctypes

    out = (ctypes.c_double * 2)()
    # soft gains stay (r >= r_nr)
    lib.sapo_effective_pd_gains(100.0, 1.0, 2e-3, 1.0, out)
    assert tuple(out) == (100.0, 1.0)
    # stiff gains are clipped so that 1/(dt (dt kp + kd)) == r_nr, keeping tau = kd/kp
    kp, kd, dt, dlt = 1e12, 1e9, 2e-3, 0.5
    lib.sapo_effective_pd_gains(kp, kd, dt, dlt, out)
    r_nr = 0.01 / (4 * np.pi**2) * dlt
    np.testing.assert_allclose(1.0 / (dt * (dt * out[0] + out[1])), r_nr, rtol=1e-12)
    np.testing.assert_allclose(out[1] / out[0], kd / kp, rtol=1e-12)
    assert lib.sapo_clamp(5.0, 2.0) == 2.0 and lib.sapo_clamp(5.0, 0.0) == 5.0
    assert lib.sapo_clamp_derivative(5.0, 2.0) == 0.0 and lib.sapo_clamp_derivative(1.0, 2.0) == 1.0
    assert lib.sapo_clamp_antiderivative(3.0, 2.0) == 2.0 * (3.0 - 1.0)
    assert lib.sapo_clamp_antiderivative(-3.0, 2.0) == -2.0 * (-3.0 + 1.0)
