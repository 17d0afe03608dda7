"""Generate tests/golden/known_answers.json: closed-form answers of the
reference's SAP formulas, computed here in plain Python without the oracle.

Projection (sim/contact_solve.py:743-921): for each regime the expected
gamma, cost and G are written out from their closed forms.  Solve cases:
a point mass resting on the ground (normal regime) and a single PD-driven DOF
(sim/contact_solve.py:490-602), whose minimizers have closed forms.

Run: python tests/golden/make_known_answers.py
"""

import json
import math
from pathlib import Path

PI = 3.141592653589793


def consts(phi0, w, mu, k, tau, dt, beta=1.0, sigma=1e-3):
    rn = max(beta * beta / (4 * PI * PI) * w, 1.0 / (dt * k * (dt + tau)))
    rt = sigma * w
    return rt, rn, -phi0 / (dt + tau)


def projection_case(name, vc, phi0, w, mu, k, tau, dt=2e-3):
    rt, rn, vhat = consts(phi0, w, mu, k, tau, dt)
    y = [-vc[0] / rt, -vc[1] / rt, (vhat - vc[2]) / rn]
    yr = math.sqrt(y[0] ** 2 + y[1] ** 2 + 1e-14)
    t = [y[0] / yr, y[1] / yr]
    zero3 = [[0.0] * 3 for _ in range(3)]
    if mu <= 1e-12:
        if y[2] > 0:
            gamma, mode = [0.0, 0.0, y[2]], 3
            G = [[0, 0, 0], [0, 0, 0], [0, 0, 1 / rn]]
        else:
            gamma, mode, G = [0.0, 0.0, 0.0], 0, zero3
    else:
        mu_hat = mu * rt / rn
        factor = 1.0 / (1.0 + mu * mu * rt / rn)
        if yr <= mu * y[2]:
            gamma, mode = list(y), 1
            G = [[1 / rt, 0, 0], [0, 1 / rt, 0], [0, 0, 1 / rn]]
        elif -mu_hat * yr < y[2] < yr / mu:
            gn = (y[2] + mu_hat * yr) * factor
            gamma, mode = [mu * gn * t[0], mu * gn * t[1], gn], 2
            P = [[t[0] * t[0], t[0] * t[1]], [t[1] * t[0], t[1] * t[1]]]
            G = [[0.0] * 3 for _ in range(3)]
            for a in range(2):
                for b in range(2):
                    G[a][b] = mu * (gn / yr * ((1.0 if a == b else 0.0) - P[a][b]) + mu_hat * factor * P[a][b]) / rt
                G[a][2] = mu * factor * t[a] / rn
                G[2][a] = mu_hat * factor * t[a] / rt
            G[2][2] = factor / rn
        else:
            gamma, mode, G = [0.0, 0.0, 0.0], 0, zero3
    cost = 0.5 * (rt * (gamma[0] ** 2 + gamma[1] ** 2) + rn * gamma[2] ** 2)
    return dict(name=name, vc=vc, phi0=phi0, w=w, mu=mu, k=k, tau=tau, dt=dt, gamma=gamma, mode=mode, cost=cost, G=G)


def main():
    cases = [
        projection_case("stiction_soft", [1e-6, -2e-6, 0.0], -1e-3, 0.5, 0.6, 1e5, 0.01),
        projection_case("stiction_rigid", [1e-7, 0.0, -1e-4], -1e-4, 0.2, 0.9, 1e10, 0.0),
        projection_case("sliding_x", [0.3, 0.0, 0.0], -1e-3, 0.5, 0.6, 1e5, 0.01),
        projection_case("sliding_xy", [0.3, 0.1, -0.01], -5e-4, 1.5, 0.3, 1e6, 0.005),
        projection_case("sliding_rigid", [0.05, -0.02, 0.0], -1e-4, 0.1, 1.0, 1e10, 0.0),
        projection_case("separating", [0.0, 0.0, 1.0], 1e-3, 0.5, 0.6, 1e5, 0.01),
        projection_case("no_contact_fast_slide", [5.0, 0.0, 0.5], 0.0, 0.5, 0.6, 1e5, 0.01),
        projection_case("frictionless_press", [0.2, 0.0, -0.01], -1e-3, 0.5, 0.0, 1e5, 0.01),
        projection_case("frictionless_apart", [0.2, 0.0, 0.5], 1e-3, 0.5, 0.0, 1e5, 0.01),
        projection_case("at_rest_penetrating", [0.0, 0.0, 0.0], -2e-3, 1.0, 0.5, 1e5, 0.01),
    ]
    # Point mass m on the ground (n = 3 translational DOFs, J = I, contact normal +z,
    # phi0 = 0, diag-Delassus w = 1/(sqrt(3) m)), starting at rest under gravity:
    # v* = (0, 0, -g dt).  Stiction/normal regime: gamma = R^-1 (vhat - vc) and
    # m (v - v*) = gamma give v_n = -m g dt R_n / (m R_n + 1), gamma_n = m g dt / (m R_n + 1).
    m, g, dt, k, tau = 2.0, 9.81, 2e-3, 1e10, 0.0
    w = 1.0 / (math.sqrt(3.0) * m)
    rt, rn, _ = consts(0.0, w, 0.8, k, tau, dt)
    vn = -m * g * dt * rn / (m * rn + 1.0)
    gn = m * g * dt / (m * rn + 1.0)
    resting = dict(m=m, g=g, dt=dt, k=k, tau=tau, w=w, mu=0.8, v=[0.0, 0.0, vn], gamma=[0.0, 0.0, gn])
    # One DOF with a PD drive (no contacts, no clamp): ell = A/2 (v-v*)^2 + dt/(2 gain) y^2,
    # y = a - gain v, gain = dt kp + kd, a = kp (q_target - q) + kd v_target.
    A, vstar, kp, kd, q, qt, vt = 1.5, 0.2, 50.0, 2.0, 0.1, 0.4, -0.3
    gain = dt * kp + kd
    a = kp * (qt - q) + kd * vt
    v_pd = (A * vstar + dt * a) / (A + dt * gain)
    pd = dict(A=A, v_star=vstar, kp=kp, kd=kd, q=q, q_target=qt, v_target=vt, dt=dt, v=v_pd)
    out = dict(projection=cases, resting_point_mass=resting, pd_single_dof=pd)
    path = Path(__file__).resolve().parent / "known_answers.json"
    path.write_text(json.dumps(out, indent=1))
    print(path)


if __name__ == "__main__":
    main()
