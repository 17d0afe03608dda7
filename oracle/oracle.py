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
    srcs = [HERE / "sap_oracle.c", HERE / "sap_free_motion.c", HERE / "sap_oracle.h", HERE.parent / "include" / "sapb.h"]
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


# ---- free motion, contact rows, integration (oracle/sap_free_motion.c) --------
_POINT = {"witness_point": 0, "contact_midpoint": 1}
_WEIGHT = {"body_inertia": 0, "diag_delassus": 1}


def _bind_free_motion(lib):
    lib.sapo_free_motion_contacts.restype = ctypes.c_int32
    lib.sapo_free_motion_contacts.argtypes = [
        ctypes.POINTER(_abi.ModelDesc), ctypes.POINTER(_abi.StepInputs), ctypes.POINTER(_abi.PrepareOptions),
        ctypes.POINTER(_abi.PrepareOutputs), ctypes.c_int32]
    lib.sapo_integrate_positions.restype = ctypes.c_int32
    lib.sapo_integrate_positions.argtypes = [ctypes.POINTER(_abi.ModelDesc)] + [ctypes.c_void_p] * 4 + [
        ctypes.c_int32, ctypes.c_void_p]


class HostModel:
    """sapb_model_desc over host copies of a models.replicate() batch."""

    def __init__(self, tpl: dict, g: dict):
        c = g["counts"]
        self.keep = {}
        d = _abi.ModelDesc()
        d.num_worlds = c["worlds"]
        d.joints_per_world, d.bodies_per_world = tpl["joints_per_world"], tpl["bodies_per_world"]
        d.dofs_per_world, d.coords_per_world = tpl["dofs_per_world"], tpl["coords_per_world"]
        d.articulations_per_world = len(tpl["articulation_start"]) - 1
        d.num_shapes = c["shapes"]

        def k(name, a, dtype):
            arr = np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=dtype)
            self.keep[name] = arr
            return arr.ctypes.data

        for name in ("joint_type", "joint_parent", "joint_child", "joint_ancestor", "joint_q_start",
                     "joint_qd_start", "joint_dof_dim", "articulation_start", "shape_body"):
            setattr(d, name, k(name, g[name], np.int32))
        for name in ("joint_axis", "joint_X_p", "joint_X_c", "joint_armature", "body_mass", "body_inertia",
                     "body_com", "gravity", "shape_material_mu", "shape_material_ke", "shape_material_tau"):
            setattr(d, name, k(name, g[name], np.float64))
        self.desc = d
        self.W, self.n, self.B = d.num_worlds, d.dofs_per_world, d.bodies_per_world


def free_motion_contacts(hm: HostModel, joint_q, joint_qd, contacts: dict, dt, max_contacts: int, *,
                         point_mode="contact_midpoint", weight_mode="diag_delassus", fallback_mu=0.0,
                         fallback_k=1.0e10, fallback_tau=0.0, threads: int = 0, want_factor: bool = False) -> dict:
    """The C restatement of sapb_free_motion_contacts on host arrays:
    joint_q (W, Q), joint_qd (W, n), contacts a models.ground_contacts-style
    dict (the FP64 mirrors are used), dt (W,)."""
    lib = load()
    if not hasattr(lib, "_fm_bound"):
        _bind_free_motion(lib)
        lib._fm_bound = True
    W, n, B, C = hm.W, hm.n, hm.B, max_contacts
    keep = {}

    def ptr(name, a, dtype):
        arr = np.ascontiguousarray(a, dtype=dtype)
        keep[name] = arr
        return arr.ctypes.data

    inp = _abi.StepInputs()
    inp.joint_q = ptr("q", joint_q, np.float64)
    inp.joint_qd = ptr("qd", joint_qd, np.float64)
    inp.dt = ptr("dt", np.broadcast_to(np.asarray(dt, np.float64), (W,)), np.float64)
    inp.contact_capacity = int(np.asarray(contacts["shape0"]).size)
    inp.contact_count = ptr("count", np.asarray(contacts["count"]).reshape(-1)[:1], np.int32)
    inp.contact_shape0 = ptr("sh0", contacts["shape0"], np.int32)
    inp.contact_shape1 = ptr("sh1", contacts["shape1"], np.int32)
    f64 = "point0d" in contacts
    inp.contact_point0 = ptr("p0", contacts["point0d" if f64 else "point0"], np.float64)
    inp.contact_point1 = ptr("p1", contacts["point1d" if f64 else "point1"], np.float64)
    inp.contact_normal = ptr("nr", contacts["normald" if f64 else "normal"], np.float64)
    inp.contact_margin0 = ptr("m0", contacts["margin0d" if f64 else "margin0"], np.float64)
    inp.contact_margin1 = ptr("m1", contacts["margin1d" if f64 else "margin1"], np.float64)
    opt = _abi.PrepareOptions()
    opt.max_contacts, opt.contact_weight_mode = C, _WEIGHT[weight_mode]
    opt.contact_point_mode = _POINT[point_mode]
    opt.fallback_mu, opt.fallback_stiffness, opt.fallback_tau_d = fallback_mu, fallback_k, fallback_tau
    res = dict(v_star=np.zeros((W, n)), vdot=np.zeros((W, n)), A=np.zeros((W, n, n)),
               jac=np.zeros((W, C, 3, n)), count=np.zeros(W, np.int32), phi0=np.zeros((W, C)),
               w=np.zeros((W, C)), mu=np.zeros((W, C)), k=np.zeros((W, C)), tau=np.zeros((W, C)),
               body0=np.full((W, C), -1, np.int32), body1=np.full((W, C), -1, np.int32),
               point=np.zeros((W, C, 3)), frame=np.zeros((W, C, 3, 3)), truncated=np.zeros(1, np.int32),
               body_q=np.zeros((W * B, 7)), vc_star=np.zeros((W, C, 3)))
    if want_factor:
        res["factor"] = np.zeros((W, n, n))
    out = _abi.PrepareOutputs()
    out.v_star, out.vdot, out.dynamics_matrix = (res[k].ctypes.data for k in ("v_star", "vdot", "A"))
    out.jacobian, out.contact_count, out.phi0 = (res[k].ctypes.data for k in ("jac", "count", "phi0"))
    out.w_eff, out.mu, out.stiffness, out.tau_d = (res[k].ctypes.data for k in ("w", "mu", "k", "tau"))
    out.body0, out.body1, out.point, out.frame = (res[k].ctypes.data for k in ("body0", "body1", "point", "frame"))
    out.truncated_count, out.body_q = res["truncated"].ctypes.data, res["body_q"].ctypes.data
    out.vc_star = res["vc_star"].ctypes.data
    if want_factor:
        out.dynamics_factor = res["factor"].ctypes.data
    st = lib.sapo_free_motion_contacts(ctypes.byref(hm.desc), ctypes.byref(inp), ctypes.byref(opt),
                                       ctypes.byref(out), int(threads))
    if st != 0:
        raise RuntimeError(f"oracle free motion failed with status {st}")
    res["truncated"] = int(res["truncated"][0])
    return res


def integrate_positions(hm: HostModel, joint_q, v_prev, v_new, dt, mode: str = "sap_euler") -> np.ndarray:
    """The C restatement of sapb_integrate_positions on host arrays."""
    lib = load()
    if not hasattr(lib, "_fm_bound"):
        _bind_free_motion(lib)
        lib._fm_bound = True
    q = np.ascontiguousarray(joint_q, np.float64)
    vp = np.ascontiguousarray(v_prev, np.float64)
    vn = np.ascontiguousarray(v_new, np.float64)
    h = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, np.float64), (hm.W,)))
    out = q.copy()
    st = lib.sapo_integrate_positions(ctypes.byref(hm.desc), q.ctypes.data, vp.ctypes.data, vn.ctypes.data,
                                      h.ctypes.data, 1 if mode == "midpoint" else 0, out.ctypes.data)
    if st != 0:
        raise RuntimeError(f"oracle integration failed with status {st}")
    return out
