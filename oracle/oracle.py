"""ctypes front end of the C oracle (oracle/sap_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (see oracle/__init__.py).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from pathlib import Path

import numpy as np

from sap_warp_b200 import _abi

HERE = Path(__file__).resolve().parent
LIB = HERE / "libsap_oracle.so"
_lock = threading.Lock()
_lib = None


def build(force: bool = False) -> Path:
    srcs = [HERE / "sap_oracle.c", HERE / "sap_oracle.h", HERE.parent / "include" / "sapb.h"]
    if force or not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
        res = subprocess.run(["make", "-C", str(HERE), "-B"], capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


class Projection(ctypes.Structure):
    _fields_ = [
        ("gamma", ctypes.c_double * 3),
        ("g", ctypes.c_double * 9),
        ("y", ctypes.c_double * 3),
        ("rt", ctypes.c_double),
        ("rn", ctypes.c_double),
        ("cost", ctypes.c_double),
        ("mode", ctypes.c_int32),
    ]


def load():
    global _lib
    with _lock:
        if _lib is None:
            build()
            lib = ctypes.CDLL(str(LIB))
            lib.sapo_contact_solve.restype = ctypes.c_int32
            lib.sapo_contact_solve.argtypes = [
                ctypes.POINTER(_abi.ContactProblem), ctypes.POINTER(_abi.SolveOptions),
                ctypes.POINTER(_abi.SolveOutputs), ctypes.c_int32,
            ]
            lib.sapo_solve_options_default.argtypes = [ctypes.POINTER(_abi.SolveOptions), ctypes.c_int32]
            lib.sapo_project_contact.argtypes = [
                ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_double, ctypes.c_double,
                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                ctypes.c_int, ctypes.POINTER(Projection),
            ]
            lib.sapo_effective_pd_gains.argtypes = [
                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)
            ]
            for name in ("sapo_clamp", "sapo_clamp_derivative", "sapo_clamp_antiderivative"):
                fn = getattr(lib, name)
                fn.restype = ctypes.c_double
                fn.argtypes = [ctypes.c_double, ctypes.c_double]
            lib.sapo_cholesky.restype = ctypes.c_int32
            lib.sapo_cholesky.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int32]
            _lib = lib
        return _lib


def options(line_search_variant: str = "monotone_decay", **overrides) -> _abi.SolveOptions:
    variant = line_search_variant
    o = _abi.SolveOptions()
    load().sapo_solve_options_default(ctypes.byref(o), _abi.LINE_SEARCH_VARIANTS[variant])
    for k, v in overrides.items():
        if v is None:
            continue
        if k in ("linear_solve_precision", "hessian_precision") and isinstance(v, str):
            v = _abi.SAPB_FP32 if v.lower() in ("fp32", "f32") else _abi.SAPB_FP64
        setattr(o, k, v)
    return o


def project(vc, phi0, w_eff, mu, k, tau_d, beta=1.0, sigma=1e-3, dt=2e-3, hessian=True) -> dict:
    p = Projection()
    arr = (ctypes.c_double * 3)(*[float(x) for x in vc])
    load().sapo_project_contact(arr, phi0, w_eff, mu, k, tau_d, beta, sigma, dt, int(hessian), ctypes.byref(p))
    return dict(
        gamma=np.array(p.gamma[:]), G=np.array(p.g[:]).reshape(3, 3), y=np.array(p.y[:]),
        rt=p.rt, rn=p.rn, cost=p.cost, mode=int(p.mode),
    )


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def solve(prob, line_search_variant: str = "monotone_decay", threads: int = 0, v_guess=None,
          v_guess_active: bool = False, dof_terms: dict | None = None, gamma0=None, **overrides) -> dict:
    """Run the oracle on a scenes.ContactProblemArrays (host).  gamma0
    (E, C, 3) or (K, E, C, 3): candidate starting impulse sets (the
    lowest-cost start among the plain one and the candidates is taken)."""
    lib = load()
    E, n, C = prob.num_envs, prob.dof_per_env, prob.max_contacts
    keep = {}

    def ptr(name, a, dtype):
        if a is None:
            return None
        arr = _c(a, dtype)
        keep[name] = arr
        return arr.ctypes.data

    P = _abi.ContactProblem()
    P.num_envs, P.dof_per_env, P.max_contacts = E, n, C
    P.num_bodies = int(np.asarray(prob.body_dof_start).size)
    P.contact_count = ptr("count", prob.contact_count, np.int32)
    P.dynamics_matrix = ptr("A", prob.dynamics_matrix, np.float64)
    P.jacobian = ptr("J", prob.jacobian, np.float64)
    P.phi0 = ptr("phi0", prob.phi0, np.float64)
    P.w_eff = ptr("w", prob.w_eff, np.float64)
    P.mu = ptr("mu", prob.mu, np.float64)
    P.stiffness = ptr("k", prob.stiffness, np.float64)
    P.tau_d = ptr("tau", prob.tau_d, np.float64)
    P.body0 = ptr("b0", prob.body0, np.int32)
    P.body1 = ptr("b1", prob.body1, np.int32)
    P.body_dof_start = ptr("bds", prob.body_dof_start, np.int32)
    P.body_dof_count = ptr("bdc", prob.body_dof_count, np.int32)
    P.v_star = ptr("vs", prob.v_star, np.float64)
    P.v0 = ptr("v0", prob.v0, np.float64)
    P.dt = ptr("dt", prob.dt, np.float64)
    P.gamma0 = ptr("gamma0", gamma0, np.float64)
    if gamma0 is not None:
        P.gamma0_count = int(np.asarray(gamma0).size // (3 * max(E * C, 1)))
    guess = None
    if v_guess is not None:
        guess = _c(v_guess, np.float64).copy()
        keep["guess"] = guess
        P.v_guess = guess.ctypes.data
        flag = np.array([1 if v_guess_active else 0], dtype=np.int32)
        keep["flag"] = flag
        P.v_guess_active = flag.ctypes.data
    if dof_terms is not None:
        D = _abi.DofTerms()
        D.has_pd = int(dof_terms.get("has_pd", 0))
        D.has_limits = int(dof_terms.get("has_limits", 0))
        jq = dof_terms.get("joint_q")
        D.joint_coord_count = int(np.asarray(jq).size) if jq is not None else 0
        types = {
            "dof_coord_index": np.int32, "dof_target_index": np.int32, "limit_supported": np.int32,
            "joint_target_mode": np.int32, "joint_target_ke": np.float32, "joint_target_kd": np.float32,
            "joint_effort_limit": np.float32, "joint_limit_lower": np.float64, "joint_limit_upper": np.float64,
            "joint_limit_ke": np.float64, "joint_limit_kd": np.float64, "joint_q": np.float64,
            "joint_target_pos": np.float32, "joint_target_vel": np.float32, "joint_act": np.float32,
        }
        for name, dt in types.items():
            setattr(D, name, ptr("dof_" + name, dof_terms.get(name), dt))
        keep["D"] = D
        P.dof = ctypes.pointer(D)
    out = dict(
        v=np.zeros(E * n), contact_gamma=np.zeros((E, max(C, 1), 3)), contact_mode=np.zeros((E, max(C, 1)), np.int32),
        cost=np.zeros(E), newton_iterations=np.zeros(E, np.int32), line_search_iterations=np.zeros(E, np.int32),
        converged=np.zeros(E, np.int32), status=np.zeros(E, np.int32), grad_norm=np.zeros(E),
        warm_start_accepted=np.zeros(E, np.int32),
    )
    O = _abi.SolveOutputs()
    for k, a in out.items():
        setattr(O, k, a.ctypes.data)
    opts = options(line_search_variant, **overrides)
    status = lib.sapo_contact_solve(ctypes.byref(P), ctypes.byref(opts), ctypes.byref(O), int(threads))
    if status != 0:
        raise RuntimeError(f"oracle solve failed with status {status}")
    if guess is not None:
        out["v_guess"] = guess
    return out
