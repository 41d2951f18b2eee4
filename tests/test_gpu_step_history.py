"""Per-step records (`tsp_b200_get_step_history`): several steps run in one tsp_b200_step call
leave one record each, oldest first, with the step counter, the step's device time and its
Jacobi iteration count, equal to what per-call statistics report for the same steps."""
import pytest

from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import SimBackendB200

pytestmark = pytest.mark.gpu


def dam():
    st, dmin, dmax, p = S.dam_32k()
    g = SimBackendB200(p)
    g.set_sim_domain_bounds(dmin, dmax)
    g.pull(st, p)
    g.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    return g, p


def test_step_history_of_one_call_matches_per_step_stats():
    g, p = dam()
    assert g.step_history() == []
    g.step(p, 6)
    h = g.step_history()
    assert [r["step"] for r in h] == [1, 2, 3, 4, 5, 6]
    assert all(r["ms"] > 0.0 and r["solverIters"] >= p.minSolverIters for r in h)
    s = g.stats()
    assert h[-1]["solverIters"] == s.solverIters and h[-1]["ms"] == pytest.approx(s.lastStepMs)
    assert g.step_history(2) == h[-2:]
    # the same steps one call each: same iteration counts (deterministic steps)
    g2, p2 = dam()
    per_call = []
    for _ in range(6):
        g2.step(p2)
        per_call.append(g2.stats().solverIters)
    assert [r["solverIters"] for r in h] == per_call
    assert [r["solverIters"] for r in g2.step_history()] == per_call
    g.close()
    g2.close()
