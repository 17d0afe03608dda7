"""Independent numpy statement of the SAP objective used by the tests.

It restates the same reference formulas as the oracle but in vectorised
numpy, so tests can check the oracle's outputs (optimality, cost, closed-form
answers) without trusting the oracle's own arithmetic.
"""

from __future__ import annotations

import numpy as np

PI = 3.141592653589793
SOFT = 1.0e-7


def contact_constants(phi0, w, mu, k, tau, beta=1.0, sigma=1.0e-3, dt=2.0e-3):
    """R_t, R_n, vhat_n (sim/contact_solve.py:793-823)."""
    w = np.where((w < 1e-12) | ~np.isfinite(w), 1e-12, w)
    rn_hard = beta * beta / (4 * PI * PI) * w
    k = np.where((k <= 0) | ~np.isfinite(k), 1.0, k)
    tau = np.maximum(tau, 0.0)
    rn = np.maximum(rn_hard, 1.0 / (dt * k * (dt + tau)))
    rt = np.maximum(sigma * w, 1e-30)
    rn = np.maximum(rn, 1e-30)
    vhat = -phi0 / (dt + tau)
    return rt, rn, vhat


def project(vc, mu, rt, rn, vhat):
    """gamma (..., 3), mode (...) of the regularized cone projection."""
    vc = np.asarray(vc, dtype=float)
    y = np.stack([-vc[..., 0] / rt, -vc[..., 1] / rt, (vhat - vc[..., 2]) / rn], -1)
    yr = np.sqrt(y[..., 0] ** 2 + y[..., 1] ** 2 + SOFT * SOFT)
    mu = np.where((mu < 0) | ~np.isfinite(mu), 0.0, mu)
    mu_hat = mu * rt / rn
    mu_tilde = mu * np.sqrt(rt / rn)
    factor = 1.0 / (1.0 + mu_tilde**2)
    gamma = np.zeros_like(y)
    mode = np.zeros(y.shape[:-1], dtype=np.int32)
    fric = mu <= 1e-12
    fl = fric & (y[..., 2] > 0)
    gamma[fl, 2] = y[fl, 2]
    mode[fl] = 3
    st = ~fric & (yr <= mu * y[..., 2])
    gamma[st] = y[st]
    mode[st] = 1
    sl = ~fric & ~st & (-mu_hat * yr < y[..., 2]) & (y[..., 2] < yr / np.where(mu > 0, mu, 1.0))
    gn = (y[..., 2] + mu_hat * yr) * factor
    t = y[..., :2] / yr[..., None]
    gamma[sl, 2] = gn[sl]
    gamma[sl, 0] = (mu * gn * t[..., 0])[sl]
    gamma[sl, 1] = (mu * gn * t[..., 1])[sl]
    mode[sl] = 2
    return gamma, mode


def contact_cost(gamma, rt, rn):
    return 0.5 * (rt * (gamma[..., 0] ** 2 + gamma[..., 1] ** 2) + rn * gamma[..., 2] ** 2)


def objective(v, A, v_star, J, phi0, w, mu, k, tau, count, dt=2.0e-3, beta=1.0, sigma=1.0e-3):
    """ell(v) and grad for ONE world without PD / limit terms.
    J: (C, 3, n); only the first `count` contacts are live."""
    J = J[:count]
    rt, rn, vhat = contact_constants(phi0[:count], w[:count], mu[:count], k[:count], tau[:count], beta, sigma, dt)
    r = v - v_star
    vc = np.einsum("crj,j->cr", J, v)
    gamma, mode = project(vc, mu[:count], rt, rn, vhat)
    ell = 0.5 * r @ A @ r + contact_cost(gamma, rt, rn).sum()
    grad = A @ r - np.einsum("crj,cr->j", J, gamma)
    return ell, grad, gamma, mode
