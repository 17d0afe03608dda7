"""Thin torch-facing wrapper over ``sapb_contact_solve`` (include/sapb.h).

Buffers are torch tensors on a CUDA device; this module only checks dtypes and
shapes, packs raw pointers into the ABI structs and launches on the current
torch stream.  It allocates nothing per call once a ``ContactSolveBuffers`` is
built, so a call can be captured in a CUDA graph.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import torch

from . import _abi
from ._lib import check, load

F64 = torch.float64
F32 = torch.float32
I32 = torch.int32


def normalize_sap_line_search_mode(value: str) -> str:
    """Canonical line-search name (sim/contact_solve.py:69-81)."""
    mode = str(value).strip().lower().replace("-", "_")
    aliases = {"monotone": "monotone_decay", "armijo": "armijo_decay", "exact": "exact_root"}
    mode = aliases.get(mode, mode)
    if mode not in _abi.LINE_SEARCH_VARIANTS:
        raise ValueError(
            f"line_search_variant must be one of {', '.join(_abi.LINE_SEARCH_VARIANTS)}, got {value!r}."
        )
    return mode


def make_options(line_search_variant: str = "monotone_decay", **overrides) -> _abi.SolveOptions:
    """SolveOptions with the reference defaults for the variant, then overrides."""
    variant = normalize_sap_line_search_mode(line_search_variant)
    opts = _abi.SolveOptions()
    load().sapb_solve_options_default(ctypes.byref(opts), _abi.LINE_SEARCH_VARIANTS[variant])
    for key, value in overrides.items():
        if value is None:
            continue
        if key in ("linear_solve_precision", "hessian_precision") and isinstance(value, str):
            value = _abi.SAPB_FP32 if value.lower() in ("fp32", "f32") else _abi.SAPB_FP64
        if not hasattr(opts, key):
            raise TypeError(f"unknown contact-solve option {key!r}")
        setattr(opts, key, value)
    return opts


def _ptr(t: torch.Tensor | None, dtype: torch.dtype | None = None, numel: int | None = None, name: str = "") -> int:
    if t is None:
        return 0
    if not t.is_cuda:
        raise TypeError(f"{name}: expected a CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name}: expected dtype {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: expected a contiguous tensor")
    if numel is not None and t.numel() < numel:
        raise ValueError(f"{name}: expected at least {numel} elements, got {t.numel()}")
    return t.data_ptr()


@dataclass
class ContactSolveBuffers:
    """Outputs and workspace for one (E, n, C) shape."""

    num_envs: int
    dof_per_env: int
    max_contacts: int
    device: torch.device
    v: torch.Tensor = field(init=False)
    contact_gamma: torch.Tensor = field(init=False)
    contact_mode: torch.Tensor = field(init=False)
    cost: torch.Tensor = field(init=False)
    newton_iterations: torch.Tensor = field(init=False)
    line_search_iterations: torch.Tensor = field(init=False)
    converged: torch.Tensor = field(init=False)
    status: torch.Tensor = field(init=False)
    grad_norm: torch.Tensor = field(init=False)
    warm_start_accepted: torch.Tensor = field(init=False)
    workspace: torch.Tensor = field(init=False)

    def __post_init__(self):
        E, n, C, dev = self.num_envs, self.dof_per_env, self.max_contacts, self.device
        self.v = torch.zeros(E * n, dtype=F64, device=dev)
        self.contact_gamma = torch.zeros(E, max(C, 1), 3, dtype=F64, device=dev)
        self.contact_mode = torch.zeros(E, max(C, 1), dtype=I32, device=dev)
        self.cost = torch.zeros(E, dtype=F64, device=dev)
        self.newton_iterations = torch.zeros(E, dtype=I32, device=dev)
        self.line_search_iterations = torch.zeros(E, dtype=I32, device=dev)
        self.converged = torch.zeros(E, dtype=I32, device=dev)
        self.status = torch.zeros(E, dtype=I32, device=dev)
        self.grad_norm = torch.zeros(E, dtype=F64, device=dev)
        self.warm_start_accepted = torch.zeros(E, dtype=I32, device=dev)
        ws = int(load().sapb_contact_solve_workspace_size(E, n, C))
        self.workspace = torch.zeros(max(ws, 16), dtype=torch.uint8, device=dev)


class DofTermArrays:
    """Device copies of the per-DOF drive and limit model (sapb_dof_terms)."""

    def __init__(self, **arrays):
        self.has_pd = int(arrays.pop("has_pd", 0))
        self.has_limits = int(arrays.pop("has_limits", 0))
        self.arrays = arrays
        self.struct = _abi.DofTerms()
        self.struct.has_pd = self.has_pd
        self.struct.has_limits = self.has_limits
        jq = arrays.get("joint_q")
        self.struct.joint_coord_count = int(jq.numel()) if jq is not None else 0
        types = {
            "dof_coord_index": I32, "dof_target_index": I32, "limit_supported": I32, "joint_target_mode": I32,
            "joint_target_ke": F32, "joint_target_kd": F32, "joint_effort_limit": F32,
            "joint_limit_lower": F64, "joint_limit_upper": F64, "joint_limit_ke": F64, "joint_limit_kd": F64,
            "joint_q": F64, "joint_target_pos": F32, "joint_target_vel": F32, "joint_act": F32,
        }
        for name, dtype in types.items():
            setattr(self.struct, name, _ptr(arrays.get(name), dtype, name=name))


def build_problem(
    *,
    num_envs: int,
    dof_per_env: int,
    max_contacts: int,
    contact_count: torch.Tensor,
    dynamics_matrix: torch.Tensor,
    jacobian: torch.Tensor,
    phi0: torch.Tensor,
    w_eff: torch.Tensor,
    mu: torch.Tensor,
    stiffness: torch.Tensor,
    tau_d: torch.Tensor | None,
    v_star: torch.Tensor,
    v0: torch.Tensor,
    dt: torch.Tensor,
    body0: torch.Tensor | None = None,
    body1: torch.Tensor | None = None,
    body_dof_start: torch.Tensor | None = None,
    body_dof_count: torch.Tensor | None = None,
    v_guess: torch.Tensor | None = None,
    v_guess_active: torch.Tensor | None = None,
    dof_terms: DofTermArrays | None = None,
    gamma0: torch.Tensor | None = None,
    world_order: torch.Tensor | None = None,
    v_candidates: torch.Tensor | None = None,
    gamma0_base: torch.Tensor | None = None,
    dynamics_factor: torch.Tensor | None = None,
    dof_count: torch.Tensor | None = None,
) -> _abi.ContactProblem:
    """sapb_contact_problem over device tensors (shapes and dtypes checked)."""
    E, n, C = num_envs, dof_per_env, max_contacts
    P = _abi.ContactProblem()
    P.num_envs, P.dof_per_env, P.max_contacts = E, n, C
    P.num_bodies = int(body_dof_start.numel()) if body_dof_start is not None else 0
    P.contact_count = _ptr(contact_count, I32, E, "contact_count")
    P.dynamics_matrix = _ptr(dynamics_matrix, F64, E * n * n, "dynamics_matrix")
    P.jacobian = _ptr(jacobian, F64, E * C * 3 * n, "jacobian")
    P.phi0 = _ptr(phi0, F64, E * C, "phi0")
    P.w_eff = _ptr(w_eff, F64, E * C, "w_eff")
    P.mu = _ptr(mu, F64, E * C, "mu")
    P.stiffness = _ptr(stiffness, F64, E * C, "stiffness")
    P.tau_d = _ptr(tau_d, F64, E * C, "tau_d")
    P.body0 = _ptr(body0, I32, E * C, "body0")
    P.body1 = _ptr(body1, I32, E * C, "body1")
    P.body_dof_start = _ptr(body_dof_start, I32, None, "body_dof_start")
    P.body_dof_count = _ptr(body_dof_count, I32, None, "body_dof_count")
    P.v_star = _ptr(v_star, F64, E * n, "v_star")
    P.v0 = _ptr(v0, F64, E * n, "v0")
    P.v_guess = _ptr(v_guess, F64, E * n, "v_guess")
    P.v_guess_active = _ptr(v_guess_active, I32, 1, "v_guess_active")
    P.dt = _ptr(dt, F64, E, "dt")
    P.gamma0 = _ptr(gamma0, F64, E * C * 3, "gamma0")
    if gamma0 is not None:
        P.gamma0_count = int(gamma0.numel() // (3 * max(E * C, 1)))
    P.world_order = _ptr(world_order, I32, E, "world_order")
    P.v_candidates = _ptr(v_candidates, F64, E * n, "v_candidates")
    if v_candidates is not None:
        P.v_candidate_count = int(v_candidates.numel() // max(E * n, 1))
    P.gamma0_base = _ptr(gamma0_base, F64, E * n, "gamma0_base")
    P.dynamics_factor = _ptr(dynamics_factor, F64, E * n * n, "dynamics_factor")
    P.dof_count = _ptr(dof_count, I32, E, "dof_count")
    if dof_terms is not None:
        P.dof = ctypes.pointer(dof_terms.struct)
    return P


def contact_solve(
    *,
    buffers: ContactSolveBuffers,
    options: _abi.SolveOptions,
    stream: torch.cuda.Stream | None = None,
    **arrays,
) -> ContactSolveBuffers:
    """Launch the fused solve; results land in `buffers` (no host sync).

    `arrays` are the keyword tensors of `build_problem` (contact_count,
    dynamics_matrix, jacobian, phi0, w_eff, mu, stiffness, tau_d, v_star, v0,
    dt and the optional body maps, v_guess, v_guess_active, dof_terms and the
    candidate starting impulses gamma0, (E, C, 3) or (K, E, C, 3), their
    base velocity gamma0_base (E*n), the candidate start velocities
    v_candidates, (E*n) or (K, E*n), the LDL^T dynamics_factor and the
    persistent kernel's world_order)."""
    lib = load()
    b = buffers
    P = build_problem(num_envs=b.num_envs, dof_per_env=b.dof_per_env, max_contacts=b.max_contacts, **arrays)
    out = _abi.SolveOutputs()
    out.v = b.v.data_ptr()
    out.contact_gamma = b.contact_gamma.data_ptr()
    out.contact_mode = b.contact_mode.data_ptr()
    out.cost = b.cost.data_ptr()
    out.newton_iterations = b.newton_iterations.data_ptr()
    out.line_search_iterations = b.line_search_iterations.data_ptr()
    out.converged = b.converged.data_ptr()
    out.status = b.status.data_ptr()
    out.grad_norm = b.grad_norm.data_ptr()
    out.warm_start_accepted = b.warm_start_accepted.data_ptr()
    s = stream if stream is not None else torch.cuda.current_stream(b.device)
    status = lib.sapb_contact_solve(
        ctypes.byref(P), ctypes.byref(options), ctypes.byref(out), b.workspace.data_ptr(), b.workspace.numel(),
        ctypes.c_void_p(s.cuda_stream),
    )
    check(status, "sapb_contact_solve")
    return buffers


def problem_to_device(prob, device) -> dict:
    """Device tensors of a scenes.ContactProblemArrays."""
    t = lambda a, dt: torch.as_tensor(a, dtype=dt).contiguous().to(device)
    return dict(
        contact_count=t(prob.contact_count, I32),
        dynamics_matrix=t(prob.dynamics_matrix, F64),
        jacobian=t(prob.jacobian, F64),
        phi0=t(prob.phi0, F64),
        w_eff=t(prob.w_eff, F64),
        mu=t(prob.mu, F64),
        stiffness=t(prob.stiffness, F64),
        tau_d=t(prob.tau_d, F64),
        body0=t(prob.body0, I32),
        body1=t(prob.body1, I32),
        body_dof_start=t(prob.body_dof_start, I32),
        body_dof_count=t(prob.body_dof_count, I32),
        v_star=t(prob.v_star, F64),
        v0=t(prob.v0, F64),
        dt=t(prob.dt, F64),
    )


def blocked_contact_solve(
    *,
    buffers: ContactSolveBuffers,
    options: _abi.SolveOptions,
    trees_per_env: int,
    tree_dofs: int = 6,
    stream: torch.cuda.Stream | None = None,
    contact_count: torch.Tensor,
    tree_mass: torch.Tensor,
    jacobian: torch.Tensor,
    contact_tree: torch.Tensor,
    phi0: torch.Tensor,
    w_eff: torch.Tensor,
    mu: torch.Tensor,
    stiffness: torch.Tensor,
    tau_d: torch.Tensor | None,
    v_star: torch.Tensor,
    v0: torch.Tensor,
    dt: torch.Tensor,
    v_guess: torch.Tensor | None = None,
    v_guess_active: torch.Tensor | None = None,
    world_order: torch.Tensor | None = None,
    gamma0: torch.Tensor | None = None,
    tree_dof_start: torch.Tensor | None = None,
) -> ContactSolveBuffers:
    """Launch the tree-blocked solve (sapb_blocked_contact_solve) for worlds of
    `trees_per_env` trees in blocks of `tree_dofs` DOFs; results land in
    `buffers` (dof_per_env = trees_per_env * tree_dofs, or the last entry of
    tree_dof_start, int32 [T+1], for trees of different sizes), no host
    sync.  gamma0 (E, C, 3): starting impulses of a candidate start
    v* + A^-1 J^T gamma0."""
    lib = load()
    b = buffers
    E, C, T, NB = b.num_envs, b.max_contacts, trees_per_env, tree_dofs
    if tree_dof_start is None and T * NB != b.dof_per_env:
        raise ValueError(f"buffers hold {b.dof_per_env} DOFs per world, not {T} trees x {NB}")
    if tree_dof_start is not None and b.dof_per_env > T * NB:
        raise ValueError(f"{T} trees of at most {NB} DOFs cannot hold {b.dof_per_env} DOFs per world")
    n = b.dof_per_env
    P = _abi.BlockedProblem()
    P.num_envs, P.trees_per_env, P.tree_dofs, P.max_contacts = E, T, NB, C
    P.tree_dof_start = _ptr(tree_dof_start, I32, T + 1, "tree_dof_start")
    P.dofs_per_world = n
    P.contact_count = _ptr(contact_count, I32, E, "contact_count")
    P.tree_mass = _ptr(tree_mass, F64, E * T * NB * NB, "tree_mass")
    P.jacobian = _ptr(jacobian, F64, E * C * 3 * 2 * NB, "jacobian")
    P.contact_tree = _ptr(contact_tree, I32, E * C * 2, "contact_tree")
    P.phi0 = _ptr(phi0, F64, E * C, "phi0")
    P.w_eff = _ptr(w_eff, F64, E * C, "w_eff")
    P.mu = _ptr(mu, F64, E * C, "mu")
    P.stiffness = _ptr(stiffness, F64, E * C, "stiffness")
    P.tau_d = _ptr(tau_d, F64, E * C, "tau_d")
    P.v_star = _ptr(v_star, F64, E * n, "v_star")
    P.v0 = _ptr(v0, F64, E * n, "v0")
    P.v_guess = _ptr(v_guess, F64, E * n, "v_guess")
    P.v_guess_active = _ptr(v_guess_active, I32, 1, "v_guess_active")
    P.dt = _ptr(dt, F64, E, "dt")
    P.world_order = _ptr(world_order, I32, E, "world_order")
    P.gamma0 = _ptr(gamma0, F64, E * C * 3, "gamma0")
    P.gamma0_count = 1 if gamma0 is not None else 0
    out = _abi.SolveOutputs()
    out.v = b.v.data_ptr()
    out.contact_gamma = b.contact_gamma.data_ptr()
    out.contact_mode = b.contact_mode.data_ptr()
    out.cost = b.cost.data_ptr()
    out.newton_iterations = b.newton_iterations.data_ptr()
    out.line_search_iterations = b.line_search_iterations.data_ptr()
    out.converged = b.converged.data_ptr()
    out.status = b.status.data_ptr()
    out.grad_norm = b.grad_norm.data_ptr()
    out.warm_start_accepted = b.warm_start_accepted.data_ptr()
    s = stream if stream is not None else torch.cuda.current_stream(b.device)
    status = lib.sapb_blocked_contact_solve(
        ctypes.byref(P), ctypes.byref(options), ctypes.byref(out), b.workspace.data_ptr(), b.workspace.numel(),
        ctypes.c_void_p(s.cuda_stream),
    )
    check(status, "sapb_blocked_contact_solve")
    return buffers


def blocked_fill_capacity(trees_per_env: int, tree_dofs: int, max_contacts: int, hessian_precision: str) -> int:
    """Off-diagonal factor blocks one world of this shape holds on chip."""
    prec = _abi.SAPB_FP32 if hessian_precision == "fp32" else _abi.SAPB_FP64
    return int(load().sapb_blocked_fill_capacity(trees_per_env, tree_dofs, max_contacts, prec))


def dense_to_blocked(arrays: dict, num_envs: int, dof_per_env: int, max_contacts: int, trees_per_env: int,
                     tree_dofs: int = 6, stream: torch.cuda.Stream | None = None,
                     tree_dof_start: torch.Tensor | None = None) -> dict:
    """Blocked tensors (tree_mass, jacobian, contact_tree) gathered on the
    device from the dense problem tensors of `build_problem`; tree_dof_start
    (int32 [T+1]) for trees of different sizes, each at most tree_dofs."""
    lib = load()
    E, C, T, NB = num_envs, max_contacts, trees_per_env, tree_dofs
    dev = arrays["dynamics_matrix"].device
    P = build_problem(num_envs=E, dof_per_env=dof_per_env, max_contacts=C, **arrays)
    tm = torch.empty(E, T, NB, NB, dtype=F64, device=dev)
    jac = torch.empty(E, C, 3, 2 * NB, dtype=F64, device=dev)
    ct = torch.empty(E, C, 2, dtype=I32, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    tds = _ptr(tree_dof_start, I32, T + 1, "tree_dof_start")
    status = lib.sapb_dense_to_blocked(ctypes.byref(P), T, NB, tds, tm.data_ptr(), jac.data_ptr(), ct.data_ptr(),
                                       ctypes.c_void_p(s.cuda_stream))
    check(status, "sapb_dense_to_blocked")
    return dict(tree_mass=tm, jacobian=jac, contact_tree=ct)


def blocked_problem_to_device(prob, device) -> dict:
    """Device tensors of a scenes.BlockedProblemArrays."""
    t = lambda a, dt: torch.as_tensor(a, dtype=dt).contiguous().to(device)
    return dict(
        contact_count=t(prob.contact_count, I32),
        tree_mass=t(prob.tree_mass, F64),
        jacobian=t(prob.jacobian, F64),
        contact_tree=t(prob.contact_tree, I32),
        phi0=t(prob.phi0, F64),
        w_eff=t(prob.w_eff, F64),
        mu=t(prob.mu, F64),
        stiffness=t(prob.stiffness, F64),
        tau_d=t(prob.tau_d, F64),
        v_star=t(prob.v_star, F64),
        v0=t(prob.v0, F64),
        dt=t(prob.dt, F64),
    )
