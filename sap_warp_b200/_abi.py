"""ctypes mirror of the C ABI in include/sapb.h.

The struct layouts here must match the header field for field; the
``test_abi_layout`` test checks sizes against the compiled library.
"""

from __future__ import annotations

import ctypes as C

SAPB_ABI_VERSION = 20

SAPB_OK = 0
SAPB_ERR_INVALID_ARGUMENT = -100
SAPB_ERR_UNSUPPORTED = -101
SAPB_ERR_CUDA = -102
SAPB_ERR_WORKSPACE_TOO_SMALL = -103
SAPB_ERR_TIMEOUT = -104

SAPB_LS_ASCENT_DIRECTION = -1
SAPB_LS_ALPHA_UNDERFLOW = -2
SAPB_LS_BAD_BRACKET = -3
SAPB_LS_BAD_GUESS = -4
SAPB_LS_ROOT_ITERATION_CAP = -5
SAPB_WORLD_FACTOR_CAPACITY = -10
SAPB_WORLD_NOT_FINITE = -11
SAPB_WORLD_NOT_SPD = -12

SAPB_CONTACT_MODE_NONE = 0
SAPB_CONTACT_MODE_STICTION = 1
SAPB_CONTACT_MODE_SLIDING = 2
SAPB_CONTACT_MODE_FRICTIONLESS = 3

SAPB_LS_MONOTONE_DECAY = 0
SAPB_LS_ARMIJO_DECAY = 1
SAPB_LS_EXACT_ROOT = 2

SAPB_FP64 = 0
SAPB_FP32 = 1

LINE_SEARCH_VARIANTS = {
    "monotone_decay": SAPB_LS_MONOTONE_DECAY,
    "armijo_decay": SAPB_LS_ARMIJO_DECAY,
    "exact_root": SAPB_LS_EXACT_ROOT,
}

_p = C.c_void_p


class SolveOptions(C.Structure):
    _fields_ = [
        ("contact_beta", C.c_double),
        ("contact_sigma", C.c_double),
        ("contact_tau_d", C.c_double),
        ("diag_shift", C.c_double),
        ("max_iterations", C.c_int32),
        ("optimality_abs_tol", C.c_double),
        ("optimality_rel_tol", C.c_double),
        ("cost_abs_tol", C.c_double),
        ("cost_rel_tol", C.c_double),
        ("line_search_max_iterations", C.c_int32),
        ("armijo_c", C.c_double),
        ("rho", C.c_double),
        ("line_search_relative_slop", C.c_double),
        ("line_search_variant", C.c_int32),
        ("linear_solve_precision", C.c_int32),
        ("hessian_precision", C.c_int32),
        ("cubic_init", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("ldlt_block", C.c_int32),
        ("skip_plain_start", C.c_int32),
        ("threads_per_cta", C.c_int32),
    ]


class DofTerms(C.Structure):
    _fields_ = [
        ("has_pd", C.c_int32),
        ("has_limits", C.c_int32),
        ("joint_coord_count", C.c_int32),
        ("dof_coord_index", _p),
        ("dof_target_index", _p),
        ("limit_supported", _p),
        ("joint_target_mode", _p),
        ("joint_target_ke", _p),
        ("joint_target_kd", _p),
        ("joint_effort_limit", _p),
        ("joint_limit_lower", _p),
        ("joint_limit_upper", _p),
        ("joint_limit_ke", _p),
        ("joint_limit_kd", _p),
        ("joint_q", _p),
        ("joint_target_pos", _p),
        ("joint_target_vel", _p),
        ("joint_act", _p),
        ("world_dof_start", _p),
    ]


class ContactProblem(C.Structure):
    _fields_ = [
        ("num_envs", C.c_int32),
        ("dof_per_env", C.c_int32),
        ("max_contacts", C.c_int32),
        ("num_bodies", C.c_int32),
        ("contact_count", _p),
        ("dynamics_matrix", _p),
        ("jacobian", _p),
        ("phi0", _p),
        ("w_eff", _p),
        ("mu", _p),
        ("stiffness", _p),
        ("tau_d", _p),
        ("body0", _p),
        ("body1", _p),
        ("body_dof_start", _p),
        ("body_dof_count", _p),
        ("v_star", _p),
        ("v0", _p),
        ("v_guess", _p),
        ("v_guess_active", _p),
        ("dt", _p),
        ("dof", C.POINTER(DofTerms)),
        ("gamma0", _p),
        ("gamma0_count", C.c_int32),
        ("dynamics_factor", _p),
        ("world_order", _p),
        ("v_candidates", _p),
        ("v_candidate_count", C.c_int32),
        ("gamma0_base", _p),
        ("dof_count", _p),
    ]


class BlockedProblem(C.Structure):
    _fields_ = [
        ("num_envs", C.c_int32),
        ("trees_per_env", C.c_int32),
        ("tree_dofs", C.c_int32),
        ("max_contacts", C.c_int32),
        ("contact_count", _p),
        ("tree_mass", _p),
        ("jacobian", _p),
        ("contact_tree", _p),
        ("phi0", _p),
        ("w_eff", _p),
        ("mu", _p),
        ("stiffness", _p),
        ("tau_d", _p),
        ("v_star", _p),
        ("v0", _p),
        ("v_guess", _p),
        ("v_guess_active", _p),
        ("dt", _p),
        ("world_order", _p),
        ("gamma0", _p),
        ("gamma0_count", C.c_int32),
        ("tree_dof_start", _p),
        ("dofs_per_world", C.c_int32),
        ("dof", C.POINTER(DofTerms)),
    ]


SAPB_SHAPE_PLANE, SAPB_SHAPE_SPHERE, SAPB_SHAPE_BOX = 0, 1, 2


class CollisionShapes(C.Structure):
    _fields_ = [
        ("num_worlds", C.c_int32),
        ("shapes_per_world", C.c_int32),
        ("num_global_shapes", C.c_int32),
        ("shape_type", _p),
        ("shape_scale", _p),
        ("shape_X_bs", _p),
        ("shape_body", _p),
        ("shape_margin", _p),
        ("gap", C.c_double),
        ("shape_collision_group", _p),
    ]


class ContactOutputs(C.Structure):
    _fields_ = [
        ("capacity", C.c_int32),
        ("count", _p),
        ("shape0", _p),
        ("shape1", _p),
        ("point0", _p),
        ("point1", _p),
        ("normal", _p),
        ("margin0", _p),
        ("margin1", _p),
    ]


class SolveOutputs(C.Structure):
    _fields_ = [
        ("v", _p),
        ("contact_gamma", _p),
        ("contact_mode", _p),
        ("cost", _p),
        ("newton_iterations", _p),
        ("line_search_iterations", _p),
        ("converged", _p),
        ("status", _p),
        ("grad_norm", _p),
        ("warm_start_accepted", _p),
    ]


SAPB_JOINT_PRISMATIC, SAPB_JOINT_REVOLUTE, SAPB_JOINT_BALL, SAPB_JOINT_FIXED = 0, 1, 2, 3
SAPB_JOINT_FREE, SAPB_JOINT_DISTANCE, SAPB_JOINT_D6 = 4, 5, 6
SAPB_WEIGHT_BODY_INERTIA, SAPB_WEIGHT_DIAG_DELASSUS = 0, 1
SAPB_POINT_WITNESS, SAPB_POINT_MIDPOINT = 0, 1
SAPB_INTEGRATE_SAP_EULER, SAPB_INTEGRATE_MIDPOINT = 0, 1


class ModelDesc(C.Structure):
    _fields_ = [
        ("num_worlds", C.c_int32),
        ("joints_per_world", C.c_int32),
        ("bodies_per_world", C.c_int32),
        ("dofs_per_world", C.c_int32),
        ("coords_per_world", C.c_int32),
        ("articulations_per_world", C.c_int32),
        ("num_shapes", C.c_int32),
        ("joint_type", _p),
        ("joint_parent", _p),
        ("joint_child", _p),
        ("joint_ancestor", _p),
        ("joint_q_start", _p),
        ("joint_qd_start", _p),
        ("joint_dof_dim", _p),
        ("articulation_start", _p),
        ("joint_axis", _p),
        ("joint_X_p", _p),
        ("joint_X_c", _p),
        ("joint_armature", _p),
        ("body_mass", _p),
        ("body_inertia", _p),
        ("body_com", _p),
        ("gravity", _p),
        ("shape_body", _p),
        ("shape_material_mu", _p),
        ("shape_material_ke", _p),
        ("shape_material_tau", _p),
        ("world_joint_start", _p),
        ("world_body_start", _p),
        ("world_dof_start", _p),
        ("world_articulation_start", _p),
        ("body_world", _p),
        ("total_joints", C.c_int32),
        ("total_bodies", C.c_int32),
        ("total_dofs", C.c_int32),
        ("total_articulations", C.c_int32),
    ]


class StepInputs(C.Structure):
    _fields_ = [
        ("joint_q", _p),
        ("joint_qd", _p),
        ("joint_f", _p),
        ("body_f", _p),
        ("dt", _p),
        ("contact_capacity", C.c_int32),
        ("contact_count", _p),
        ("contact_shape0", _p),
        ("contact_shape1", _p),
        ("contact_point0", _p),
        ("contact_point1", _p),
        ("contact_normal", _p),
        ("contact_margin0", _p),
        ("contact_margin1", _p),
    ]


class PrepareOptions(C.Structure):
    _fields_ = [
        ("max_contacts", C.c_int32),
        ("contact_weight_mode", C.c_int32),
        ("contact_point_mode", C.c_int32),
        ("fallback_mu", C.c_double),
        ("fallback_stiffness", C.c_double),
        ("fallback_tau_d", C.c_double),
        ("tree_blocked", C.c_int32),
        ("factor_new_contacts_only", C.c_int32),
        ("tree_dofs", C.c_int32),
    ]


class PrepareOutputs(C.Structure):
    _fields_ = [
        ("v_star", _p),
        ("vdot", _p),
        ("dynamics_matrix", _p),
        ("jacobian", _p),
        ("contact_count", _p),
        ("phi0", _p),
        ("w_eff", _p),
        ("mu", _p),
        ("stiffness", _p),
        ("tau_d", _p),
        ("body0", _p),
        ("body1", _p),
        ("point", _p),
        ("frame", _p),
        ("truncated_count", _p),
        ("body_q", _p),
        ("dynamics_factor", _p),
        ("vc_star", _p),
        ("tree_mass", _p),
        ("contact_tree", _p),
        ("contact_source", _p),
        ("history", _p),
        ("v_start", _p),
        ("qd_slots", _p),
    ]


SAPB_MLP_INPUTS = 12
SAPB_MLP_INPUTS_PADDED = 16
SAPB_MLP_HIDDEN = 128
SAPB_MLP_OUTPUTS = 3
SAPB_MLP_PARAM_COUNT = 35075
SAPB_MLP_PACKED_COUNT = 35200
SAPB_MLP_BIAS_COUNT = 387


class WarmstartNorm(C.Structure):
    _fields_ = [
        ("feature_mean", C.c_float * SAPB_MLP_INPUTS),
        ("feature_inv_std", C.c_float * SAPB_MLP_INPUTS),
        ("output_scale", C.c_float * SAPB_MLP_OUTPUTS),
        ("output_shift", C.c_float * SAPB_MLP_OUTPUTS),
    ]


class MlpTrainBuffers(C.Structure):
    _fields_ = [("act", _p), ("pre", _p), ("dy", _p), ("loss", _p)]


class AdamOptions(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("weight_decay", C.c_float)]


SAPB_WARM_START_PREVIOUS_VELOCITY = 0
SAPB_WARM_START_PREVIOUS_IMPULSES = 1
SAPB_WARM_START_LEARNED = 2
SAPB_WORK_ORDER_INDEX = 0
SAPB_WORK_ORDER_PREVIOUS_ITERATIONS = 1


class StepNetwork(C.Structure):
    _fields_ = [("packed", _p), ("bias", _p), ("norm", WarmstartNorm), ("feature_tau_d", C.c_double),
                ("impulse_tau_d", C.c_double)]


class StepOptions(C.Structure):
    _fields_ = [("prepare", PrepareOptions), ("solve", SolveOptions), ("position_integration", C.c_int32),
                ("warm_start", C.c_int32), ("work_order", C.c_int32), ("impulse_history", C.c_int32),
                ("network", C.POINTER(StepNetwork))]


class StepIO(C.Structure):
    _fields_ = [("inp", StepInputs), ("dof", C.POINTER(DofTerms)), ("joint_q_out", _p), ("joint_qd_out", _p)]


class StepTail(C.Structure):
    _fields_ = [("joint_q_in", _p), ("v_prev", _p), ("v_new", _p), ("dt", _p), ("mode", C.c_int32),
                ("qd_public", C.c_int32), ("joint_q_out", _p), ("joint_qd_out", _p), ("body_q_out", _p),
                ("body_qd_out", _p)]


class ContactHistory(C.Structure):
    _fields_ = [("num_envs", C.c_int32), ("max_contacts", C.c_int32), ("num_flat", C.c_int32),
                ("contact_count", _p), ("contact_source", _p), ("flat_shape0", _p), ("flat_shape1", _p),
                ("flat_point1", _p), ("key_shape", _p), ("key_point", _p), ("key_count", _p), ("gamma_prev", _p),
                ("gamma_hist", _p), ("has_history", _p), ("order", C.c_int32), ("gamma_older", _p),
                ("gamma_start", _p)]


# name -> (restype, argtypes) of every symbol include/sapb.h declares.
EXPORTS = {
    "sapb_solve_options_default": (None, [C.POINTER(SolveOptions), C.c_int32]),
    "sapb_abi_version": (C.c_int32, []),
    "sapb_measure_fma_rate": (C.c_int32, [C.c_int32, C.c_int32, C.POINTER(C.c_double), _p]),
    "sapb_step_options_default": (None, [C.POINTER(StepOptions)]),
    "sapb_create": (C.c_int32, [C.POINTER(ModelDesc), C.POINTER(StepOptions), C.POINTER(_p)]),
    "sapb_step": (C.c_int32, [_p, C.POINTER(StepIO), _p]),
    "sapb_get_status": (C.c_int32, [_p, _p, _p, _p, _p]),
    "sapb_step_solve_outputs": (C.c_int32, [_p, C.POINTER(SolveOutputs)]),
    "sapb_destroy": (None, [_p]),
    "sapb_world_order": (C.c_int32, [_p, C.c_int32, _p, _p]),
    "sapb_contact_history_update": (C.c_int32, [C.POINTER(ContactHistory), _p]),
    "sapb_step_tail_launch": (C.c_int32, [C.POINTER(ModelDesc), C.POINTER(StepTail), _p]),
    "sapb_contact_solve_workspace_size": (C.c_size_t, [C.c_int32, C.c_int32, C.c_int32]),
    "sapb_contact_solve_occupancy": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "sapb_contact_solve_occupancy_threads": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "sapb_contact_solve_ldlt_blocks": (C.c_int32, [C.c_int32, C.POINTER(C.c_int32), C.c_int32]),
    "sapb_contact_solve": (
        C.c_int32,
        [C.POINTER(ContactProblem), C.POINTER(SolveOptions), C.POINTER(SolveOutputs), _p, C.c_size_t, _p],
    ),
    "sapb_contact_solve_noalloc": (
        C.c_int32, [C.POINTER(ContactProblem), C.POINTER(SolveOptions), C.POINTER(SolveOutputs), _p]
    ),
    "sapb_last_error": (C.c_char_p, []),
    "sapb_blocked_fill_capacity": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "sapb_blocked_solve_workspace_size": (C.c_size_t, [C.c_int32, C.c_int32, C.c_int32]),
    "sapb_blocked_contact_solve": (
        C.c_int32,
        [C.POINTER(BlockedProblem), C.POINTER(SolveOptions), C.POINTER(SolveOutputs), _p, C.c_size_t, _p],
    ),
    "sapb_dense_to_blocked": (C.c_int32, [C.POINTER(ContactProblem), C.c_int32, C.c_int32, _p, _p, _p, _p, _p]),
    "sapb_blocked_tree_block": (C.c_int32, [C.c_int32]),
    "sapb_prepare_workspace_size": (C.c_size_t, [C.POINTER(ModelDesc), C.c_int32]),
    "sapb_free_motion_contacts": (
        C.c_int32,
        [C.POINTER(ModelDesc), C.POINTER(StepInputs), C.POINTER(PrepareOptions), C.POINTER(PrepareOutputs), _p,
         C.c_size_t, _p],
    ),
    "sapb_public_to_sap": (C.c_int32, [C.POINTER(ModelDesc), _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "sapb_sap_to_public_velocity": (C.c_int32, [C.POINTER(ModelDesc), _p, _p, _p, _p]),
    "sapb_eval_fk": (C.c_int32, [C.POINTER(ModelDesc), _p, _p, _p, _p, _p]),
    "sapb_contacts_workspace_size": (C.c_size_t, [C.POINTER(CollisionShapes)]),
    "sapb_generate_contacts": (
        C.c_int32, [C.POINTER(CollisionShapes), _p, C.POINTER(ContactOutputs), _p, C.c_size_t, _p]
    ),
    "sapb_integrate_positions": (
        C.c_int32, [C.POINTER(ModelDesc), _p, _p, _p, _p, C.c_int32, _p, _p]
    ),
    "sapb_mlp_param_count": (C.c_int32, []),
    "sapb_mlp_packed_count": (C.c_int32, []),
    "sapb_mlp_bias_count": (C.c_int32, []),
    "sapb_mlp_train_buffer_sizes": (C.c_int32, [C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "sapb_mlp_pack": (C.c_int32, [_p, _p, _p, _p]),
    "sapb_mlp_forward": (C.c_int32, [_p, _p, _p, C.c_int32, _p, _p]),
    "sapb_mlp_forward_train": (C.c_int32, [_p, _p, _p, _p, C.c_int32, C.POINTER(MlpTrainBuffers), _p, _p]),
    "sapb_mlp_backward": (C.c_int32, [_p, _p, C.c_int32, C.POINTER(MlpTrainBuffers), _p, _p]),
    "sapb_mlp_adam": (C.c_int32, [_p, _p, _p, _p, C.POINTER(AdamOptions), C.c_int32, _p, _p, _p]),
    "sapb_mlp_error": (C.c_int32, [_p]),
    "sapb_mlp_test_hooks": (C.c_int32, [C.c_int32, C.c_int32]),
    "sapb_warmstart_features": (
        C.c_int32, [C.POINTER(ContactProblem), _p, _p, _p, C.POINTER(WarmstartNorm), C.c_double, _p, _p, _p]
    ),
    "sapb_warmstart_impulses": (
        C.c_int32, [C.POINTER(ContactProblem), _p, _p, _p, C.POINTER(WarmstartNorm), C.POINTER(SolveOptions), _p, _p]
    ),
    "sapb_warmstart_active_tiles": (C.c_int32, [C.POINTER(ContactProblem), _p, _p, _p]),
    "sapb_mlp_forward_tiles": (C.c_int32, [_p, _p, _p, C.c_int32, _p, _p, _p]),
}


def bind(lib: C.CDLL) -> C.CDLL:
    """Attach restype/argtypes for every exported symbol; raises if one is missing."""
    for name, (restype, argtypes) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    return lib
