"""The C-ABI library loads without a GPU, exports every symbol include/sapb.h
declares, and the ctypes mirror matches the header's struct layouts."""

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from sap_warp_b200 import _abi
from sap_warp_b200.build import LIB_PATH, build_library

ROOT = Path(__file__).resolve().parents[1]
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(sapb_[a-z0-9_]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    build_library()
    return _abi.bind(ctypes.CDLL(str(LIB_PATH)))


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert "sapb_contact_solve" in names
    for name in names:
        assert hasattr(lib, name), name
    assert names <= set(_abi.EXPORTS), names - set(_abi.EXPORTS)


def test_no_compute_entry_points_without_gpu(lib):
    assert lib.sapb_abi_version() == _abi.SAPB_ABI_VERSION
    o = _abi.SolveOptions()
    lib.sapb_solve_options_default(ctypes.byref(o), _abi.SAPB_LS_EXACT_ROOT)
    assert o.line_search_max_iterations == 100 and o.cost_rel_tol == 1e-15 and o.rho == 0.8
    lib.sapb_solve_options_default(ctypes.byref(o), _abi.SAPB_LS_MONOTONE_DECAY)
    assert o.cost_rel_tol == 5e-3 and o.cost_abs_tol == 0.0
    assert lib.sapb_contact_solve_workspace_size(4096, 35, 32) >= 4
    # argument errors are reported before any CUDA call
    assert lib.sapb_contact_solve(None, None, None, None, 0, None) == _abi.SAPB_ERR_INVALID_ARGUMENT
    assert lib.sapb_blocked_contact_solve(None, None, None, None, 0, None) == _abi.SAPB_ERR_INVALID_ARGUMENT
    assert lib.sapb_blocked_fill_capacity(64, 6, 448, _abi.SAPB_FP64) > 100
    assert lib.sapb_blocked_fill_capacity(64, 6, 448, _abi.SAPB_FP32) > 100
    assert lib.sapb_blocked_fill_capacity(64, 5, 448, _abi.SAPB_FP64) == 0
    # block sizes of trees of different sizes: the smallest built block that holds them
    from sap_warp_b200.solver import tree_block_for
    for nt in range(-1, 15):
        assert lib.sapb_blocked_tree_block(nt) == tree_block_for(nt)
    assert [tree_block_for(k) for k in (1, 6, 7, 8, 12, 13)] == [6, 6, 7, 12, 12, 0]
    assert lib.sapb_blocked_fill_capacity(24, 7, 256, _abi.SAPB_FP64) > 20
    assert lib.sapb_blocked_fill_capacity(16, 12, 128, _abi.SAPB_FP32) > 10
    assert b"null" in lib.sapb_last_error()
    assert lib.sapb_mlp_param_count() == _abi.SAPB_MLP_PARAM_COUNT
    assert lib.sapb_mlp_packed_count() == _abi.SAPB_MLP_PACKED_COUNT
    assert lib.sapb_mlp_bias_count() == _abi.SAPB_MLP_BIAS_COUNT
    a, p = ctypes.c_int64(), ctypes.c_int64()
    assert lib.sapb_mlp_train_buffer_sizes(300, ctypes.byref(a), ctypes.byref(p)) == _abi.SAPB_OK
    assert a.value == p.value == 3 * 3 * 128 * 128
    assert lib.sapb_mlp_forward(None, None, None, 4, None, None) == _abi.SAPB_ERR_INVALID_ARGUMENT
    assert lib.sapb_warmstart_features(None, None, None, None, None, 0.0, None, None, None) == \
        _abi.SAPB_ERR_INVALID_ARGUMENT
    # the whole-step handle, the world order and the FMA-rate probe reject bad arguments before any CUDA call
    so = _abi.StepOptions()
    lib.sapb_step_options_default(ctypes.byref(so))
    assert so.prepare.max_contacts == 128 and so.solve.line_search_variant == _abi.SAPB_LS_ARMIJO_DECAY
    assert so.work_order == _abi.SAPB_WORK_ORDER_PREVIOUS_ITERATIONS and so.impulse_history == 3
    assert lib.sapb_create(None, ctypes.byref(so), None) == _abi.SAPB_ERR_INVALID_ARGUMENT
    # option checks that come before any device access (the model's arrays are never read here)
    md = _abi.ModelDesc()
    md.num_worlds, md.joints_per_world, md.bodies_per_world, md.dofs_per_world = 2, 1, 1, 6
    md.coords_per_world, md.articulations_per_world = 7, 1
    md.joint_child = md.joint_qd_start = md.joint_dof_dim = md.articulation_start = 16  # never dereferenced
    h = ctypes.c_void_p()
    so.warm_start = _abi.SAPB_WARM_START_LEARNED  # without a network
    assert lib.sapb_create(ctypes.byref(md), ctypes.byref(so), ctypes.byref(h)) == _abi.SAPB_ERR_INVALID_ARGUMENT
    assert b"network" in lib.sapb_last_error() and not h.value
    so.warm_start = 7
    assert lib.sapb_create(ctypes.byref(md), ctypes.byref(so), ctypes.byref(h)) == _abi.SAPB_ERR_INVALID_ARGUMENT
    so.warm_start = _abi.SAPB_WARM_START_PREVIOUS_VELOCITY
    so.solve.threads_per_cta = 64  # checked by the solve entry point
    assert lib.sapb_contact_solve_occupancy_threads(35, 32, _abi.SAPB_FP32, _abi.SAPB_LS_ARMIJO_DECAY, 64) == \
        _abi.SAPB_ERR_INVALID_ARGUMENT
    assert lib.sapb_step(None, None, None) == _abi.SAPB_ERR_INVALID_ARGUMENT
    assert lib.sapb_get_status(None, None, None, None, None) == _abi.SAPB_ERR_INVALID_ARGUMENT
    lib.sapb_destroy(None)
    assert lib.sapb_world_order(None, 4, None, None) == _abi.SAPB_ERR_INVALID_ARGUMENT
    assert lib.sapb_world_order(None, 0, None, None) == _abi.SAPB_OK
    rate = ctypes.c_double()
    assert lib.sapb_measure_fma_rate(7, 16, ctypes.byref(rate), None) == _abi.SAPB_ERR_INVALID_ARGUMENT


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "sapb.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(sapb_solve_options),"
        " sizeof(sapb_dof_terms), sizeof(sapb_contact_problem), sizeof(sapb_solve_outputs),"
        " offsetof(sapb_contact_problem, dof), offsetof(sapb_solve_options, cubic_init),"
        " sizeof(sapb_model_desc), sizeof(sapb_step_inputs), sizeof(sapb_prepare_options),"
        " sizeof(sapb_prepare_outputs)); printf(\"%zu %zu %zu %zu\\n\", sizeof(sapb_warmstart_norm),"
        " sizeof(sapb_mlp_train_buffers), sizeof(sapb_adam_options), offsetof(sapb_contact_problem, gamma0));"
        " printf(\"%zu %zu\\n\", sizeof(sapb_blocked_problem), offsetof(sapb_blocked_problem, world_order));"
        " printf(\"%zu %zu %zu %zu\\n\", sizeof(sapb_step_options), offsetof(sapb_step_options, work_order),"
        " sizeof(sapb_step_io), offsetof(sapb_step_io, joint_qd_out));"
        " printf(\"%zu %zu %zu %zu\\n\", sizeof(sapb_contact_history), offsetof(sapb_contact_history, order),"
        " offsetof(sapb_contact_history, gamma_start), offsetof(sapb_step_options, impulse_history));"
        " printf(\"%zu %zu %zu %zu %zu\\n\", sizeof(sapb_step_network), offsetof(sapb_step_network, impulse_tau_d),"
        " offsetof(sapb_step_options, network), offsetof(sapb_blocked_problem, tree_dof_start),"
        " offsetof(sapb_dof_terms, world_dof_start));"
        " return 0;}\n"
    )
    exe = tmp_path / "sizes"
    cc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
    subprocess.run([cc, "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_abi.SolveOptions), ctypes.sizeof(_abi.DofTerms), ctypes.sizeof(_abi.ContactProblem),
            ctypes.sizeof(_abi.SolveOutputs), _abi.ContactProblem.dof.offset, _abi.SolveOptions.cubic_init.offset,
            ctypes.sizeof(_abi.ModelDesc), ctypes.sizeof(_abi.StepInputs), ctypes.sizeof(_abi.PrepareOptions),
            ctypes.sizeof(_abi.PrepareOutputs), ctypes.sizeof(_abi.WarmstartNorm),
            ctypes.sizeof(_abi.MlpTrainBuffers), ctypes.sizeof(_abi.AdamOptions), _abi.ContactProblem.gamma0.offset,
            ctypes.sizeof(_abi.BlockedProblem), _abi.BlockedProblem.world_order.offset,
            ctypes.sizeof(_abi.StepOptions), _abi.StepOptions.work_order.offset, ctypes.sizeof(_abi.StepIO),
            _abi.StepIO.joint_qd_out.offset, ctypes.sizeof(_abi.ContactHistory), _abi.ContactHistory.order.offset,
            _abi.ContactHistory.gamma_start.offset, _abi.StepOptions.impulse_history.offset,
            ctypes.sizeof(_abi.StepNetwork), _abi.StepNetwork.impulse_tau_d.offset, _abi.StepOptions.network.offset,
            _abi.BlockedProblem.tree_dof_start.offset, _abi.DofTerms.world_dof_start.offset]
    assert got == want
