"""The whole SolverSAP step captured in a CUDA graph: replays reproduce the
eager rollout bit for bit (the step is deterministic: slots are re-ranked,
reductions have a fixed order, each world is solved by one block)."""

import pytest
import torch

from sap_warp_b200 import models
from sap_warp_b200.runtime import SapState
from sap_warp_b200.solver import SolverSAP

pytestmark = pytest.mark.gpu


def pair(state):
    return (SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone()),
            SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone()))


@pytest.mark.parametrize("warm_start,precision", [("previous_velocity", "fp64"), ("learned", "fp32")])
def test_graph_replay_matches_eager_steps(cuda_device, warm_start, precision):
    model, state, control, contacts, _ = models.rollout_scene("humanoid", 256, 7, cuda_device)
    kw = dict(max_rigid_contact=32, contact_preset_variant="drake", hessian_precision=precision, warm_start=warm_start)
    eager, graphed = SolverSAP(model, **kw), SolverSAP(model, **kw)
    ea, eb = pair(state)
    ga, gb = pair(state)
    graph = graphed.capture_steps(ga, gb, control, contacts, 2.0e-3, warmup=1)  # 2 eager warm-up steps
    eager.step(ea, eb, control, contacts, 2.0e-3)  # the two warm-up steps of the capture
    eager.step(eb, ea, control, contacts, 2.0e-3)
    for _ in range(3):
        graph.replay()
        eager.step(ea, eb, control, contacts, 2.0e-3)
        eager.step(eb, ea, control, contacts, 2.0e-3)
    torch.cuda.synchronize()
    assert torch.equal(ga.joint_q, ea.joint_q) and torch.equal(ga.joint_qd, ea.joint_qd)
    assert bool(graphed.contact_solve.converged_env.all())
    del graph


def test_learned_fp32_rollouts_repeat_bit_for_bit(cuda_device):
    """Two solvers stepping the same 4096 worlds (learned warm start, FP32
    factor: the fastest factor, so the one where a shared-memory race in the
    blocked LDL^T would show first) give identical trajectories."""
    def run():
        model, state, control, contacts, _ = models.rollout_scene("humanoid", 4096, 20240, cuda_device)
        solver = SolverSAP(model, max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32",
                           warm_start="learned")
        a, b = pair(state)
        out = []
        for _ in range(40):
            solver.step(a, b, control, contacts, 2.0e-3)
            out.append(b.joint_qd.clone())
            a, b = b, a
        return out
    r1, r2 = run(), run()
    first = next((k for k in range(len(r1)) if not torch.equal(r1[k], r2[k])), None)
    assert first is None, f"the rollouts part at step {first}"


def test_host_step_graph_matches_eager_steps(cuda_device):
    """capture_host_steps: state and contacts from pinned host memory each
    step, the new state back to the host; its replays reproduce eager steps
    bit for bit, with the second contact set really used by the second step
    of each pair (a set with every contact moved away gives other results)."""
    from sap_warp_b200.runtime import SapContacts

    model, state, control, contacts, _ = models.rollout_scene("humanoid", 256, 11, cuda_device)
    kw = dict(max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32", warm_start="learned")
    names = [k for k in vars(contacts) if isinstance(getattr(contacts, k), torch.Tensor)]
    far = SapContacts(**{k: getattr(contacts, k).clone() for k in names})
    far.rigid_contact_point0[:, 2] -= 1.0  # separated by a metre: no contact force
    far.rigid_contact_point0d[:, 2] -= 1.0
    sets = (contacts, far)
    host_sets = tuple(SapContacts(**{k: getattr(c, k).cpu().pin_memory() for k in names}) for c in sets)
    host_state = {"joint_q": state.joint_q.cpu().pin_memory(), "joint_qd": state.joint_qd.cpu().pin_memory()}

    hs = SolverSAP(model, **kw)
    ha, hb = pair(state)
    graph = hs.capture_host_steps(host_state, host_sets, ha, hb, control, 2.0e-3, warmup=1)
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()

    es = SolverSAP(model, **kw)
    ea, eb = pair(state)
    for _ in range(4):  # the warm-up pair and three replays
        es.step(ea, eb, control, sets[0], 2.0e-3)
        es.step(eb, ea, control, sets[1], 2.0e-3)
    torch.cuda.synchronize()
    assert torch.equal(host_state["joint_q"], ea.joint_q.cpu())
    assert torch.equal(host_state["joint_qd"], ea.joint_qd.cpu())
    ref = SolverSAP(model, **kw)
    ra, rb = pair(state)
    for _ in range(8):
        ref.step(ra, rb, control, contacts, 2.0e-3)
        ra, rb = rb, ra
    assert not torch.equal(ra.joint_qd, ea.joint_qd)
    del graph
