"""Fluid-rigid coupling on the GPU against the oracle (ReduceRigidParticleForcesToBody,
PredictRigidBodies, IntegrateRigidBodies: source/simulation/CPU/backend/cpu_backend.cpp:
2009-2303; rigid force accumulations: sph_solver.cpp:1151, 1717).

Body sums and body integration run in FP64 on both sides, per-particle forces in FP32;
the differences are the FP32 summation order of the per-particle terms and the distances of
the SPH sweeps (hardware reciprocal square root on the GPU, IEEE square root in the oracle).
Tolerances:
|gpu - oracle| <= rtol * (|oracle| + max|oracle|), rtol stated per quantity.
"""
import numpy as np
import pytest

from oracle import OracleBackend
from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import SimBackendB200

pytestmark = pytest.mark.gpu

BODY_FIELDS = (("xCM", 1e-6), ("yCM", 1e-6), ("zCM", 1e-6),
               ("xVelRB", 2e-3), ("yVelRB", 2e-3), ("zVelRB", 2e-3),
               ("xOmegaRB", 2e-3), ("yOmegaRB", 2e-3), ("zOmegaRB", 2e-3),
               ("xAngMomRB", 2e-3), ("yAngMomRB", 2e-3), ("zAngMomRB", 2e-3))


def close(a, b, rtol, what):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.max(np.abs(b)) if b.size else 0.0
    err = np.abs(a - b)
    assert np.all(err <= rtol * (np.abs(b) + scale) + 1e-30), f"{what}: max err {err.max():.3e}, scale {scale:.3e}"


def cubes_pair(fp64=False):
    st, dmin, dmax, p = S.floating_cubes()
    g, o = SimBackendB200(p), OracleBackend(p, fp64=fp64)
    for be in (g, o):
        be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)
        be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    return g, o, p, st


def test_gpu_rigid_volumes_match_oracle():
    g, o, p, st = cubes_pair()
    gs, os_ = g.push(), o.push()
    assert np.array_equal(gs.idR, os_.idR), "rigid particles keep their storage order"
    close(gs.volR, os_.volR, 1e-6, "volR")
    close(gs.psiR, os_.psiR, 1e-6, "psiR")


@pytest.mark.parametrize("fp64", [False, True])
def test_gpu_rigid_steps_match_oracle(fp64):
    """Five coupled steps: identical Jacobi iteration counts, identical fluid order, body
    state and rigid-particle world positions within tolerance of the FP32 oracle and of the
    FP64 oracle."""
    g, o, p, st = cubes_pair(fp64)
    for k in range(5):
        g.step(p)
        o.step(p)
        assert g.stats().solverIters == o.stats().solverIters, f"step {k}"
    gs, os_ = g.push(), o.push()
    if not fp64:
        assert np.array_equal(gs.idF, os_.idF)
    for name, rtol in BODY_FIELDS:
        close(getattr(gs, name), getattr(os_, name), rtol, name)
    for r in range(3):
        for c in range(3):
            n = f"a{r}{c}"
            assert np.max(np.abs(getattr(gs, n).astype(np.float64) - getattr(os_, n))) <= 1e-5, n
    for n in ("xPosR", "yPosR", "zPosR"):
        close(getattr(gs, n), getattr(os_, n), 1e-6, n)
    og, oo = np.argsort(gs.idF), np.argsort(os_.idF)
    close(gs.densityF[og], os_.densityF[oo], 1e-4, "densityF")
    close(gs.yVelF[og], os_.yVelF[oo], 5e-3, "yVelF")


def test_gpu_rigid_forces_match_oracle():
    """Per-particle fluid->rigid forces and the FP64 body force/torque sums of one step."""
    g, o, p, st = cubes_pair()
    g.step(p)
    o.step(p)
    close(g.read_field(abi.FIELD_FORCE_R), o.read_field(abi.FIELD_FORCE_R), 2e-3, "rigid particle forces")
    close(g.read_field(abi.FIELD_BODY_FT), o.read_field(abi.FIELD_BODY_FT), 2e-3, "body force/torque")


def test_gpu_rigid_free_fall_known_answer():
    """A lone cube (no fluid, no walls) falls as v_k = k dt g, y_k = y_0 + dt^2 g k(k+1)/2."""
    from test_oracle_rigid import check_free_fall, lone_cube
    from turbospharticles_b200.params import dam_params
    p = dam_params(0.02, 1e-3)
    check_free_fall(SimBackendB200(p), p, lone_cube(p))


# ---- rigid contact solver (SolveRigidContacts, rigid_solver.cpp:602-799)
def test_gpu_contact_idle_without_contact():
    from test_oracle_rigid import lone_cube
    from turbospharticles_b200.params import dam_params
    p = dam_params(0.02, 1e-3)
    g = SimBackendB200(p)
    g.pull(lone_cube(p), p)
    g.step(p)
    r = g.contact_report()
    assert r.solverIters == 0 and r.converged == 1 and r.nContacts == 0


def test_gpu_contact_pair_conserves_momentum():
    from test_oracle_rigid import pressed_pair, run_pair
    from turbospharticles_b200.params import dam_params
    p = dam_params(0.02, 1e-3)
    p.gravity = (0.0, 0.0, 0.0)
    st = pressed_pair(p)
    out, reports = run_pair(SimBackendB200(p), p, st)
    o_out, o_rep = run_pair(OracleBackend(p), p, st)
    assert all(abs(a.solverIters - b.solverIters) <= 1 for a, b in zip(reports, o_rep))
    assert reports[0].nContacts == o_rep[0].nContacts
    m = st.massRB.astype(np.float64)
    px = float(np.sum(m * out.xVelRB))
    assert abs(px) <= 1e-5 * float(np.max(np.abs(m * out.xVelRB)))
    assert out.xVelRB[0] < 0.0 < out.xVelRB[1]
    close(out.xVelRB, o_out.xVelRB, 2e-3, "separation velocities vs oracle")


@pytest.mark.parametrize("fp64", [False, True])
def test_gpu_contact_matches_oracle(fp64):
    """Stacked cubes pressed into the floor and each other: per-step contact iteration counts
    (within one of the oracle's), the contact set of the first step, and the body states after
    four steps against the FP32 and the FP64 oracle."""
    st, dmin, dmax, p = S.stacked_cubes()
    g, o = SimBackendB200(p), OracleBackend(p, fp64=fp64)
    for be in (g, o):
        be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)
        be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    iters_g, iters_o = [], []
    for k in range(4):
        g.step(p)
        o.step(p)
        rg, ro = g.contact_report(), o.contact_report()
        if k == 0:
            assert rg.nContactBoundary == ro.nContactBoundary
            assert rg.nContacts == ro.nContacts
        iters_g.append(rg.solverIters)
        iters_o.append(ro.solverIters)
    assert max(iters_o) > 0
    assert all(abs(a - b) <= 1 for a, b in zip(iters_g, iters_o)), (iters_g, iters_o)
    gs, os_ = g.push(), o.push()
    for n, tol in (("xCM", 1e-5), ("yCM", 1e-4), ("zCM", 1e-5), ("xVelRB", 2e-2), ("yVelRB", 2e-2),
                   ("zOmegaRB", 2e-2)):
        close(getattr(gs, n), getattr(os_, n), tol, n)
