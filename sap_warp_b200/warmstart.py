"""Learned warm start of the SAP contact solve.

A per-contact MLP (12 -> 128 -> 128 -> 128 -> 3, GELU, BF16 weights and
activations, FP32 accumulation) predicts starting impulses gamma0 from each
contact's inputs; the solve maps them to v_L = v* + A^-1 J^T gamma0 and starts
Newton from v_L only if its cost is below that of the plain start, so the
plain solve stays both fallback and judge and every world still converges to
the same tolerance.  Inference, training (forward, backward, Adam) and the
feature / impulse maps run in the sapb_mlp_* / sapb_warmstart_* kernels
(tcgen05 tensor cores for the hidden layers).

Nothing here has a counterpart in the reference: its warm start is the
previous step's velocity (sim/solver_sap.py:1441-1451), which this module
composes with (the plain start it competes against is v_guess when active).

Network inputs of a contact slot (raw): phi0; J_c v* in the contact frame
(t1, t2, n); the world-up component of the contact normal (1 when unknown);
mu; log10(stiffness); tau_d; dt; w_eff * gamma_prev (t1, t2, n; 0 when no
previous impulses are given).  The network predicts a correction
w_eff * (y* - gamma_prev) (velocity units), y* being SAP's unprojected impulse
-R^-1 (vc - vhat) at the converged FP64 solution; the impulse map projects
gamma_prev + correction / w_eff with the solve's regularized cone projection,
so separated contacts (y_n << 0) start at exactly zero impulse.  Inputs and
targets are standardised with the statistics of the training set, which
travel with the weights.
"""

from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi
from ._lib import check, load
from ._solve import ContactSolveBuffers, build_problem, contact_solve, make_options, problem_to_device

F32, F64, I32, I16 = torch.float32, torch.float64, torch.int32, torch.int16
IN, IN_PAD, HID, OUT = _abi.SAPB_MLP_INPUTS, _abi.SAPB_MLP_INPUTS_PADDED, _abi.SAPB_MLP_HIDDEN, _abi.SAPB_MLP_OUTPUTS
PARAM_COUNT = _abi.SAPB_MLP_PARAM_COUNT
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "warmstart_humanoid.npz")

# (name, shape) of the FP32 master parameter vector, in order.
PARAM_LAYOUT = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)),
                ("b3", (HID,)), ("W4", (OUT, HID)), ("b4", (OUT,))]


def _stream(device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _dev_ptr(t: torch.Tensor, dtype, numel: int, name: str) -> int:
    if not t.is_cuda or t.dtype != dtype or not t.is_contiguous() or t.numel() < numel:
        raise ValueError(f"{name}: expected a contiguous CUDA {dtype} tensor with >= {numel} elements")
    return t.data_ptr()


def init_params(seed: int = 0) -> np.ndarray:
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases, output layer x0.1."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in PARAM_LAYOUT:
        fan_in = IN if name in ("W1", "b1") else HID
        a = rng.uniform(-1.0, 1.0, size=shape) / math.sqrt(fan_in)
        if name in ("W4", "b4"):
            a *= 0.1
        parts.append(a.astype(np.float32).reshape(-1))
    out = np.concatenate(parts)
    assert out.size == PARAM_COUNT
    return out


@dataclass
class FeatureNorm:
    """Standardisation of the 12 raw inputs and of the 3 targets."""

    mean: np.ndarray
    inv_std: np.ndarray
    out_scale: np.ndarray
    out_shift: np.ndarray

    @classmethod
    def identity(cls) -> "FeatureNorm":
        return cls(np.zeros(IN, np.float32), np.ones(IN, np.float32), np.ones(OUT, np.float32),
                   np.zeros(OUT, np.float32))

    @classmethod
    def from_data(cls, raw: np.ndarray, u: np.ndarray) -> "FeatureNorm":
        """Constant inputs (std ~ 0) get inv_std 0: they carry no information."""
        raw = np.asarray(raw, np.float64)
        u = np.asarray(u, np.float64)
        mean, std = raw.mean(0), raw.std(0)
        inv = np.where(std > 1e-6 * np.maximum(1.0, np.abs(mean)), 1.0 / np.maximum(std, 1e-30), 0.0)
        return cls(mean.astype(np.float32), inv.astype(np.float32), np.maximum(u.std(0), 1e-12).astype(np.float32),
                   u.mean(0).astype(np.float32))

    def struct(self) -> _abi.WarmstartNorm:
        s = _abi.WarmstartNorm()
        for i in range(IN):
            s.feature_mean[i] = float(self.mean[i])
            s.feature_inv_std[i] = float(self.inv_std[i])
        for j in range(OUT):
            s.output_scale[j] = float(self.out_scale[j])
            s.output_shift[j] = float(self.out_shift[j])
        return s

    def encode(self, raw: torch.Tensor) -> torch.Tensor:
        """(N, 12) FP32 raw inputs -> (N, 16) BF16 bit patterns (int16), the
        kernels' input rows (same arithmetic as the features kernel)."""
        mean = torch.as_tensor(self.mean, device=raw.device)
        inv = torch.as_tensor(self.inv_std, device=raw.device)
        x = torch.zeros(raw.shape[0], IN_PAD, dtype=torch.bfloat16, device=raw.device)
        x[:, :IN] = ((raw - mean) * inv).to(torch.bfloat16)
        return x.view(I16).contiguous()

    def targets(self, u: torch.Tensor) -> torch.Tensor:
        scale = torch.as_tensor(self.out_scale, device=u.device)
        shift = torch.as_tensor(self.out_shift, device=u.device)
        return ((u - shift) / scale).to(F32).contiguous()


class TrainBuffers:
    """Saved forward state of one training batch (sapb_mlp_train_buffers)."""

    def __init__(self, rows: int, device):
        a, p = ctypes.c_int64(), ctypes.c_int64()
        check(load().sapb_mlp_train_buffer_sizes(rows, ctypes.byref(a), ctypes.byref(p)),
              "sapb_mlp_train_buffer_sizes")
        self.rows = rows
        self.act = torch.zeros(a.value, dtype=I16, device=device)
        self.pre = torch.zeros(p.value, dtype=F32, device=device)
        self.dy = torch.zeros(rows, OUT, dtype=F32, device=device)
        self.loss = torch.zeros(1, dtype=F32, device=device)
        self.struct = _abi.MlpTrainBuffers(self.act.data_ptr(), self.pre.data_ptr(), self.dy.data_ptr(),
                                           self.loss.data_ptr())


class WarmStartMLP:
    """FP32 master parameters, Adam moments and the BF16 operand images."""

    def __init__(self, device, params: np.ndarray | None = None, seed: int = 0):
        self.device = torch.device(device)
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        if p.size != PARAM_COUNT:
            raise ValueError(f"expected {PARAM_COUNT} parameters, got {p.size}")
        self.params = torch.as_tensor(p.copy()).to(self.device).contiguous()
        self.grad = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.packed = torch.zeros(_abi.SAPB_MLP_PACKED_COUNT, dtype=I16, device=self.device)
        self.bias = torch.zeros(_abi.SAPB_MLP_BIAS_COUNT, dtype=F32, device=self.device)
        self.step = 0
        self.pack()

    def pack(self) -> None:
        check(load().sapb_mlp_pack(self.params.data_ptr(), self.packed.data_ptr(), self.bias.data_ptr(),
                                   _stream(self.device)), "sapb_mlp_pack")

    def forward(self, x: torch.Tensor, y: torch.Tensor | None = None,
                tile_active: torch.Tensor | None = None) -> torch.Tensor:
        """y = MLP(x); with tile_active (int32 per 128-row tile), only the
        tiles whose flag is nonzero are computed (the others' rows of y are
        left as they are)."""
        rows = x.shape[0]
        xp = _dev_ptr(x, I16, rows * IN_PAD, "x")
        if y is None:
            y = torch.empty(rows, OUT, dtype=F32, device=self.device)
        yp = _dev_ptr(y, F32, rows * OUT, "y")
        if tile_active is None:
            check(load().sapb_mlp_forward(self.packed.data_ptr(), self.bias.data_ptr(), xp, rows, yp,
                                          _stream(self.device)), "sapb_mlp_forward")
        else:
            tp = _dev_ptr(tile_active, torch.int32, (rows + 127) // 128, "tile_active")
            check(load().sapb_mlp_forward_tiles(self.packed.data_ptr(), self.bias.data_ptr(), xp, rows, yp, tp,
                                                _stream(self.device)), "sapb_mlp_forward_tiles")
        return y

    def forward_train(self, x: torch.Tensor, target: torch.Tensor, buf: TrainBuffers,
                      y: torch.Tensor | None = None) -> None:
        rows = x.shape[0]
        if rows > buf.rows:
            raise ValueError("batch larger than the training buffers")
        check(load().sapb_mlp_forward_train(
            self.packed.data_ptr(), self.bias.data_ptr(), _dev_ptr(x, I16, rows * IN_PAD, "x"),
            _dev_ptr(target, F32, rows * OUT, "target"), rows, ctypes.byref(buf.struct),
            None if y is None else _dev_ptr(y, F32, rows * OUT, "y"), _stream(self.device)), "sapb_mlp_forward_train")

    def backward(self, x: torch.Tensor, buf: TrainBuffers) -> None:
        rows = x.shape[0]
        check(load().sapb_mlp_backward(self.packed.data_ptr(), _dev_ptr(x, I16, rows * IN_PAD, "x"), rows,
                                       ctypes.byref(buf.struct), self.grad.data_ptr(), _stream(self.device)),
              "sapb_mlp_backward")

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8,
             weight_decay: float = 0.0) -> None:
        self.step += 1
        opt = _abi.AdamOptions(lr, beta1, beta2, eps, weight_decay)
        check(load().sapb_mlp_adam(self.params.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
                                   self.v.data_ptr(), ctypes.byref(opt), self.step, self.packed.data_ptr(),
                                   self.bias.data_ptr(), _stream(self.device)), "sapb_mlp_adam")

    def train_step(self, x: torch.Tensor, target: torch.Tensor, buf: TrainBuffers, lr: float, **adam) -> torch.Tensor:
        """One Adam step on the mean squared error; returns the batch's summed
        squared error (device tensor, no host sync)."""
        buf.loss.zero_()
        self.grad.zero_()
        self.forward_train(x, target, buf)
        self.backward(x, buf)
        self.adam(lr, **adam)
        return buf.loss

    def check_error(self) -> None:
        """Raises if a bounded wait inside an MLP kernel gave up (syncs)."""
        check(load().sapb_mlp_error(_stream(self.device)), "sapb_mlp kernels")


class LearnedWarmStart:
    """Trained network + standardisation: gamma0 for a stage-2 problem.
    contact_beta / contact_sigma / tau_fallback are the solve's
    regularization, used to project the predicted unprojected impulses."""

    def __init__(self, mlp: WarmStartMLP, norm: FeatureNorm, tau_fallback: float = 0.0, contact_beta: float = 1.0,
                 contact_sigma: float = 1.0e-3):
        self.mlp = mlp
        self.norm = norm
        self.norm_struct = norm.struct()
        self.tau_fallback = float(tau_fallback)
        self.set_regularization(contact_beta, contact_sigma, tau_fallback)
        self._bufs: dict = {}

    def set_regularization(self, contact_beta: float, contact_sigma: float, tau_fallback: float) -> None:
        self.tau_fallback = float(tau_fallback)
        self.solve_options = make_options("armijo_decay", contact_beta=float(contact_beta),
                                          contact_sigma=float(contact_sigma), contact_tau_d=float(tau_fallback))

    @property
    def device(self):
        return self.mlp.device

    def buffers(self, num_envs: int, max_contacts: int) -> dict:
        key = (num_envs, max_contacts)
        if key not in self._bufs:
            slots = num_envs * max_contacts
            self._bufs[key] = dict(
                x=torch.zeros(slots, IN_PAD, dtype=I16, device=self.device),
                y=torch.zeros(slots, OUT, dtype=F32, device=self.device),
                tiles=torch.zeros((slots + 127) // 128, dtype=torch.int32, device=self.device),
                gamma0=torch.zeros(num_envs, max_contacts, 3, dtype=F64, device=self.device))
        return self._bufs[key]

    def predict(self, *, num_envs: int, dof_per_env: int, max_contacts: int, normal_up: torch.Tensor | None = None,
                gamma_prev: torch.Tensor | None = None, vc_star: torch.Tensor | None = None,
                out: torch.Tensor | None = None, has_history: torch.Tensor | None = None,
                **arrays) -> torch.Tensor:
        """gamma0 (E, C, 3) FP64 on the device (into `out` if given):
        features -> MLP -> impulses on the current stream, no host sync, no
        allocation after the first call for a shape.  With has_history
        ((E, C) int32: the slot's contact carries gamma_prev from the
        previous step), those slots keep gamma_prev and the network predicts
        only the new contacts (tiles of 128 rows without one are skipped)."""
        E, C = num_envs, max_contacts
        b = self.buffers(E, C)
        g_out = b["gamma0"] if out is None else out
        P = build_problem(num_envs=E, dof_per_env=dof_per_env, max_contacts=C, **arrays)
        lib, s = load(), _stream(self.device)
        nu = 0 if normal_up is None else _dev_ptr(normal_up, F64, E * C, "normal_up")
        gp = 0 if gamma_prev is None else _dev_ptr(gamma_prev, F64, E * C * 3, "gamma_prev")
        vc = 0 if vc_star is None else _dev_ptr(vc_star, F64, E * C * 3, "vc_star")
        check(lib.sapb_warmstart_features(ctypes.byref(P), nu, gp, vc, ctypes.byref(self.norm_struct),
                                          self.tau_fallback, b["x"].data_ptr(), None, s), "sapb_warmstart_features")
        hh = 0 if has_history is None else _dev_ptr(has_history, torch.int32, E * C, "has_history")
        if has_history is None:
            self.mlp.forward(b["x"], b["y"])
        else:
            check(lib.sapb_warmstart_active_tiles(ctypes.byref(P), hh, b["tiles"].data_ptr(), s),
                  "sapb_warmstart_active_tiles")
            self.mlp.forward(b["x"], b["y"], tile_active=b["tiles"])
        check(lib.sapb_warmstart_impulses(ctypes.byref(P), b["y"].data_ptr(), gp, hh, ctypes.byref(self.norm_struct),
                                          ctypes.byref(self.solve_options), _dev_ptr(g_out, F64, E * C * 3, "out"), s),
              "sapb_warmstart_impulses")
        return g_out

    # ---- persistence ------------------------------------------------------------
    def save(self, path: str, **meta) -> None:
        np.savez(path, params=self.mlp.params.cpu().numpy(), mean=self.norm.mean, inv_std=self.norm.inv_std,
                 out_scale=self.norm.out_scale, out_shift=self.norm.out_shift, tau_fallback=self.tau_fallback,
                 **{f"meta_{k}": np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, device="cuda") -> "LearnedWarmStart":
        z = np.load(path)
        norm = FeatureNorm(z["mean"], z["inv_std"], z["out_scale"], z["out_shift"])
        return cls(WarmStartMLP(device, params=z["params"]), norm, float(z["tau_fallback"]))


def raw_features(arrays: dict, num_envs: int, dof_per_env: int, max_contacts: int,
                 normal_up: torch.Tensor | None = None, gamma_prev: torch.Tensor | None = None,
                 tau_fallback: float = 0.0) -> torch.Tensor:
    """(E*C, 12) FP32 raw inputs of every slot (dead slots zero)."""
    E, C = num_envs, max_contacts
    dev = arrays["jacobian"].device
    raw = torch.zeros(E * C, IN, dtype=F32, device=dev)
    P = build_problem(num_envs=E, dof_per_env=dof_per_env, max_contacts=C, **arrays)
    nu = 0 if normal_up is None else _dev_ptr(normal_up, F64, E * C, "normal_up")
    gp = 0 if gamma_prev is None else _dev_ptr(gamma_prev, F64, E * C * 3, "gamma_prev")
    check(load().sapb_warmstart_features(ctypes.byref(P), nu, gp, None, None, tau_fallback, None, raw.data_ptr(),
                                         _stream(dev)), "sapb_warmstart_features")
    return raw


def unprojected_targets(arrays: dict, v: torch.Tensor, num_envs: int, dof_per_env: int, max_contacts: int,
                        contact_beta: float = 1.0, contact_sigma: float = 1.0e-3, tau_fallback: float = 0.0):
    """(E*C, 3) u = w_eff * y of every slot: y = -R^-1 (J_c v - vhat), SAP's
    unprojected impulse at the velocity v (sim/contact_solve.py:797-870), with
    R_t = sigma w, R_n = max(beta^2 w / (4 pi^2), 1 / (dt k (dt + tau)))."""
    E, n, C = num_envs, dof_per_env, max_contacts
    J = arrays["jacobian"].reshape(E, C, 3, n)
    vc = torch.einsum("ecrj,ej->ecr", J, v.reshape(E, n))
    w = arrays["w_eff"].reshape(E, C).clamp(min=1e-12)
    tau = arrays["tau_d"].reshape(E, C) if arrays.get("tau_d") is not None else torch.full_like(w, tau_fallback)
    tau = tau.clamp(min=0.0)
    k = arrays["stiffness"].reshape(E, C)
    k = torch.where(k > 0, k, torch.ones_like(k))
    dt = arrays["dt"].reshape(E, 1)
    rt = (contact_sigma * w).clamp(min=1e-30)
    rn = torch.maximum(contact_beta ** 2 / (4.0 * math.pi ** 2) * w, 1.0 / (dt * k * (dt + tau))).clamp(min=1e-30)
    vhat = -arrays["phi0"].reshape(E, C) / (dt + tau)
    y = torch.stack([-vc[..., 0] / rt, -vc[..., 1] / rt, (vhat - vc[..., 2]) / rn], -1)
    return (w[..., None] * y).reshape(E * C, 3)


def solver_dataset(problems, device, line_search_variant: str = "armijo_decay"):
    """(raw inputs (N, 12), targets u = w_eff * y* (N, 3)) of every live
    contact of the given scenes.ContactProblemArrays, y* the unprojected
    impulse at the converged FP64 GPU solve (reference tolerances)."""
    raws, us = [], []
    opts = make_options(line_search_variant)
    for prob in problems:
        E, n, C = prob.num_envs, prob.dof_per_env, prob.max_contacts
        arrays = problem_to_device(prob, device)
        nu = None if prob.normal_up is None else torch.as_tensor(prob.normal_up, dtype=F64).to(device).contiguous()
        buf = ContactSolveBuffers(E, n, C, torch.device(device))
        contact_solve(**arrays, buffers=buf, options=opts)
        raw = raw_features(arrays, E, n, C, normal_up=nu)
        live = (torch.arange(C, device=device)[None, :] < arrays["contact_count"][:, None]).reshape(-1)
        u = unprojected_targets(arrays, buf.v, E, n, C)
        raws.append(raw[live])
        us.append(u[live].to(F32))
    return torch.cat(raws), torch.cat(us)


def rollout_dataset(kind: str, worlds: int, seeds, steps: int, device, *, every: int = 1,
                    hessian_precision: str = "fp64", contact_preset_variant: str = "drake"):
    """(raw inputs (N, 12), targets u = w_eff * y (N, 3)) of the live
    contacts along SolverSAP trajectories (reference warm start, FP64, the
    given contact preset): at
    step k the inputs carry gamma_prev = the impulses of step k-1 in the same
    slot (slot order is canonical, so a persistent contact keeps its slot),
    the targets are the unprojected impulses y at step k's converged
    velocity.  Every `every`-th step."""
    from . import models
    from .runtime import SapState
    from .solver import SolverSAP

    raws, us = [], []
    for seed in seeds:
        model, state, control, con, _ = models.rollout_scene(kind, worlds, seed, device)
        solver = SolverSAP(model, max_rigid_contact=32, hessian_precision=hessian_precision,
                           contact_preset_variant=contact_preset_variant)
        other = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(),
                         body_q=state.body_q.clone(), body_f=state.body_f.clone())
        W, n, C = solver.view.W, solver.view.n, solver.max_rigid_contact
        gamma_prev = torch.zeros(W, C, 3, dtype=F64, device=device)
        normal_up = torch.zeros(W, C, dtype=F64, device=device)
        for k in range(steps):
            solver.step(state, other, control, con, 2.0e-3)
            if k % every == 0:
                cr = solver.last_contact_jacobian_result
                normal_up.copy_(cr.contact_env_R_WC[..., 2, 2])
                arrays = dict(contact_count=cr.contact_env_count, dynamics_matrix=cr.dynamics_matrix_env,
                              jacobian=cr.contact_env_jacobian, phi0=cr.contact_env_phi0, w_eff=cr.contact_env_w_eff,
                              mu=cr.contact_env_mu, stiffness=cr.contact_env_stiffness, tau_d=cr.contact_env_tau_d,
                              v_star=solver.contact_jacobian.v_star, v0=solver.contact_jacobian.v_star,
                              dt=solver.contact_jacobian.dt_world)
                raw = raw_features(arrays, W, n, C, normal_up=normal_up, gamma_prev=gamma_prev)
                cnt = cr.contact_env_count.clamp(max=C)
                live = (torch.arange(C, device=device)[None, :] < cnt[:, None]).reshape(-1)
                u = unprojected_targets(arrays, solver.contact_solve.v_flat, W, n, C,
                                        solver.contact_solve.contact_beta, solver.contact_solve.contact_sigma)
                raws.append(raw[live])
                us.append(u[live].to(F32))
            gamma_prev.copy_(solver.contact_solve.contact_gamma)
            state, other = other, state
    return torch.cat(raws), torch.cat(us)


def site_rollout_dataset(kind: str, worlds: int, seeds, steps: int, device, *, hessian_precision: str = "fp64",
                         contact_preset_variant: str = "drake"):
    """(raw inputs (N, 12), targets u = w_eff * y (N, 3)) of the NEW contacts
    (no contact with the same identity at the previous step) along SolverSAP
    trajectories of models.site_scene, whose contacts are regenerated from
    the pose every step: the rows the learned start's network predicts when
    it serves new contacts only (their gamma_prev input is zero).  Targets:
    the unprojected impulses y at the step's converged velocity."""
    from . import models
    from .collision import ContactGenerator
    from .runtime import SapState
    from .solver import SolverSAP

    raws, us = [], []
    for seed in seeds:
        model, state, control, shapes, _ = models.site_scene(kind, worlds, seed, device)
        solver = SolverSAP(model, max_rigid_contact=32, hessian_precision=hessian_precision,
                           contact_preset_variant=contact_preset_variant, warm_start="previous_impulses")
        gen = ContactGenerator(shapes, solver.view, capacity=worlds * 32, gap=1.0e-3)
        other = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(),
                         body_q=state.body_q.clone(), body_f=state.body_f.clone())
        W, n, C = solver.view.W, solver.view.n, solver.max_rigid_contact
        normal_up = torch.zeros(W, C, dtype=F64, device=device)
        for k in range(steps):
            solver.step(state, other, control, gen.generate(state.joint_q), 2.0e-3)
            cr = solver.last_contact_jacobian_result
            normal_up.copy_(cr.contact_env_R_WC[..., 2, 2])
            arrays = dict(contact_count=cr.contact_env_count, dynamics_matrix=cr.dynamics_matrix_env,
                          jacobian=cr.contact_env_jacobian, phi0=cr.contact_env_phi0, w_eff=cr.contact_env_w_eff,
                          mu=cr.contact_env_mu, stiffness=cr.contact_env_stiffness, tau_d=cr.contact_env_tau_d,
                          v_star=solver.contact_jacobian.v_star, v0=solver.contact_jacobian.v_star,
                          dt=solver.contact_jacobian.dt_world)
            raw = raw_features(arrays, W, n, C, normal_up=normal_up)
            cnt = cr.contact_env_count.clamp(max=C)
            live = torch.arange(C, device=device)[None, :] < cnt[:, None]
            new = (live & (solver.has_history == 0)).reshape(-1)
            u = unprojected_targets(arrays, solver.contact_solve.v_flat, W, n, C,
                                    solver.contact_solve.contact_beta, solver.contact_solve.contact_sigma)
            raws.append(raw[new])
            us.append(u[new].to(F32))
            state, other = other, state
    return torch.cat(raws), torch.cat(us)


def residual_targets(raw: torch.Tensor, u: torch.Tensor, clip_quantile: float = 0.005) -> torch.Tensor:
    """w_eff * (y* - gamma_prev): the targets u minus the w-scaled previous
    impulses carried in raw input columns 9..11, each component clipped to
    its [q, 1-q] quantile range (separated contacts have arbitrarily negative
    y_n, and every value beyond the range projects the same way)."""
    r = (u - raw[:, 9:12]).contiguous()
    if clip_quantile > 0.0 and r.shape[0] > 0:
        k = min(r.shape[0], 1 << 20)
        sample = r[torch.randperm(r.shape[0], device=r.device)[:k]]
        lo = torch.quantile(sample, clip_quantile, dim=0)
        hi = torch.quantile(sample, 1.0 - clip_quantile, dim=0)
        r = torch.maximum(torch.minimum(r, hi), lo)
    return r


def train(mlp: WarmStartMLP, raw: torch.Tensor, u: torch.Tensor, norm: FeatureNorm, steps: int = 4000,
          batch: int = 8192, lr: float = 2e-3, lr_final: float = 5e-5, seed: int = 0, log_every: int = 200):
    """Adam on the standardised targets with a cosine learning-rate decay;
    returns [(step, mean squared error of the batch)]."""
    x_all = norm.encode(raw)
    t_all = norm.targets(residual_targets(raw, u))
    N = x_all.shape[0]
    gen = torch.Generator(device=mlp.device)
    gen.manual_seed(seed)
    buf = TrainBuffers(batch, mlp.device)
    log = []
    for k in range(steps):
        idx = torch.randint(0, N, (batch,), generator=gen, device=mlp.device)
        xb, tb = x_all[idx].contiguous(), t_all[idx].contiguous()
        lr_k = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * k / max(steps - 1, 1)))
        loss = mlp.train_step(xb, tb, buf, lr_k)
        if log_every and (k % log_every == 0 or k == steps - 1):
            log.append((k, float(loss.item()) / (3 * batch)))
    mlp.check_error()
    return log


def default_training_problems(humanoid_seeds=range(100, 125), quadruped_seeds=range(200, 210), worlds: int = 4096):
    """Solver-generated training scenes: the 35-DOF humanoid batch (8-32
    contacts) and the 18-DOF quadruped batch (4-16 contacts) at seeds disjoint
    from the benchmark's and the tests'."""
    from . import scenes

    for s in humanoid_seeds:
        yield scenes.humanoid_contact_problem(worlds, seed=s)
    for s in quadruped_seeds:
        yield scenes.quadruped_contact_problem(worlds, seed=s)


def _main():
    import argparse
    import time

    ap = argparse.ArgumentParser(description="Train the warm-start MLP on solver-generated contacts.")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--humanoid-seeds", type=int, default=4)
    ap.add_argument("--quadruped-seeds", type=int, default=2)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--rollout-steps", type=int, default=80)
    ap.add_argument("--rollout-every", type=int, default=2)
    a = ap.parse_args()
    dev = torch.device("cuda", 0)
    t0 = time.time()
    parts = [rollout_dataset("humanoid", 4096, range(100, 100 + a.humanoid_seeds), a.rollout_steps, dev,
                             every=a.rollout_every),
             rollout_dataset("quadruped", 4096, range(200, 200 + a.quadruped_seeds), a.rollout_steps, dev,
                             every=a.rollout_every)]
    raw = torch.cat([p[0] for p in parts])
    u = torch.cat([p[1] for p in parts])
    t1 = time.time()
    norm = FeatureNorm.from_data(raw.cpu().numpy(), residual_targets(raw, u).cpu().numpy())
    mlp = WarmStartMLP(dev, seed=a.seed)
    log = train(mlp, raw, u, norm, steps=a.steps, batch=a.batch, lr=a.lr, seed=a.seed)
    torch.cuda.synchronize()
    t2 = time.time()
    for k, l in log:
        print(f"step {k:6d}  mse {l:.5f}")
    ws = LearnedWarmStart(mlp, norm)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    ws.save(a.out, contacts=raw.shape[0], steps=a.steps, batch=a.batch, final_mse=log[-1][1])
    print(f"contacts {raw.shape[0]}  data {t1 - t0:.1f} s  train {t2 - t1:.1f} s  -> {a.out}")


if __name__ == "__main__":
    _main()
