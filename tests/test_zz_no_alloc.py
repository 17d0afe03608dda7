"""The allocation-free contact-solve entry point, through the C ABI.

sapb_contact_solve_noalloc serves callers that cannot allocate device memory
(a plugin whose host runtime owns every device allocation, or a binding with
no device allocator): it takes no workspace and uses a fixed array compiled
into the library.  This file is collected last so that a run stopping at the
first failure has already run every other test; it must also pass alone in a
fresh process.  The check: two calls in a row match the workspace entry
point's results on the same inputs.  The solve is deterministic (fixed
reduction orders, no atomics in the arithmetic), so they match bit for bit.
"""

import ctypes

import numpy as np
import pytest
import torch

from sap_warp_b200 import _abi, scenes
from sap_warp_b200._lib import load
from sap_warp_b200._solve import ContactSolveBuffers, contact_solve, make_options, problem_to_device

pytestmark = pytest.mark.gpu


def _pack(t, E, n, C):
    P = _abi.ContactProblem()
    P.num_envs, P.dof_per_env, P.max_contacts = E, n, C
    P.num_bodies = t["body_dof_start"].numel()
    for name in ("contact_count", "dynamics_matrix", "jacobian", "phi0", "w_eff", "mu", "stiffness", "tau_d",
                 "body0", "body1", "body_dof_start", "body_dof_count", "v_star", "v0", "dt"):
        setattr(P, name, t[name].data_ptr())
    return P


def _outputs(E, n, C, dev):
    bufs = dict(
        v=torch.zeros(E * n, dtype=torch.float64, device=dev),
        contact_gamma=torch.zeros(E, C, 3, dtype=torch.float64, device=dev),
        contact_mode=torch.zeros(E, C, dtype=torch.int32, device=dev),
        cost=torch.zeros(E, dtype=torch.float64, device=dev),
        newton_iterations=torch.zeros(E, dtype=torch.int32, device=dev),
        line_search_iterations=torch.zeros(E, dtype=torch.int32, device=dev),
        converged=torch.zeros(E, dtype=torch.int32, device=dev),
        status=torch.zeros(E, dtype=torch.int32, device=dev),
        grad_norm=torch.zeros(E, dtype=torch.float64, device=dev),
    )
    O = _abi.SolveOutputs()
    for k, v in bufs.items():
        setattr(O, k, v.data_ptr())
    return bufs, O


def test_noalloc_entry_point_matches_workspace_entry_point():
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    lib = load()
    prob = scenes.humanoid_contact_problem(512, seed=31)
    E, n, C = prob.num_envs, prob.dof_per_env, prob.max_contacts
    t = problem_to_device(prob, dev)
    ref = ContactSolveBuffers(E, n, C, dev)
    opts = make_options("armijo_decay")
    contact_solve(**t, buffers=ref, options=opts)
    torch.cuda.synchronize()
    P = _pack(t, E, n, C)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        bufs, O = _outputs(E, n, C, dev)
        status = lib.sapb_contact_solve_noalloc(ctypes.byref(P), ctypes.byref(opts), ctypes.byref(O),
                                                ctypes.c_void_p(stream.cuda_stream))
        assert status == _abi.SAPB_OK, lib.sapb_last_error()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(bufs["v"].cpu().numpy(), ref.v.cpu().numpy(), err_msg=f"call {call}")
        np.testing.assert_array_equal(bufs["contact_gamma"].cpu().numpy(), ref.contact_gamma.cpu().numpy(),
                                      err_msg=f"call {call}")
        np.testing.assert_array_equal(bufs["cost"].cpu().numpy(), ref.cost.cpu().numpy(), err_msg=f"call {call}")
        np.testing.assert_array_equal(bufs["contact_mode"].cpu().numpy(), ref.contact_mode.cpu().numpy())
        np.testing.assert_array_equal(bufs["converged"].cpu().numpy(), ref.converged.cpu().numpy())
        np.testing.assert_array_equal(bufs["newton_iterations"].cpu().numpy(), ref.newton_iterations.cpu().numpy())
