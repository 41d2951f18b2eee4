"""Oracle rigid-body path on the CPU: free-fall known answer of the body integrator
(PredictRigidBodies / IntegrateRigidBodies, source/simulation/CPU/backend/cpu_backend.cpp:
2174-2303: v += dt * F/m, x += dt * v, with F = m g when no fluid touches the body) and the
FP32 oracle's coupled body state against the FP64 oracle (the error statement of FP32)."""
import numpy as np
import pytest

from oracle import OracleBackend
from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.params import dam_params


def lone_cube(p):
    """One hollow cube far from anything (no fluid, no walls)."""
    box = S.OBB((1.0, 2.0, 3.0), (0.2, 0.2, 0.2))
    local, body = S.rigid_hollow_box(box, p, 800.0)
    st = S.UniversalSimState(0, 0, local[0].shape[0], 1, p.restDensity)
    st.xPosRelR[:], st.yPosRelR[:], st.zPosRelR[:] = local
    st.bodyIdR[:] = 0
    st.psiR[:] = p.massB
    st.volR[:] = np.float32(p.massB / p.restDensity)
    st.xCM[0], st.yCM[0], st.zCM[0] = body["center"]
    st.massRB[0], st.massInvRB[0] = body["mass"], body["massInv"]
    st.iBodyInv00[0], st.iBodyInv11[0], st.iBodyInv22[0] = body["iBodyInv"]
    for r in range(3):
        for c in range(3):
            getattr(st, f"a{r}{c}")[0] = body["A"][r, c]
    st.rigidParticleCountRB[0] = st.N_R
    return st


def free_fall_expected(y0, g, dt, n):
    v, y = 0.0, float(y0)
    for _ in range(n):
        v += dt * g
        y += dt * v
    return v, y


def check_free_fall(be, p, st, n=7):
    be.pull(st, p)
    be.step(p, n) if n > 1 else be.step(p)
    out = be.push()
    v, y = free_fall_expected(st.yCM[0], p.gravity[1], p.timeStep, n)
    assert abs(out.yVelRB[0] - v) <= 1e-6 * abs(v)
    assert abs(out.yCM[0] - y) <= 1e-6 * abs(y)
    assert out.xVelRB[0] == 0 and out.zVelRB[0] == 0
    assert out.xOmegaRB[0] == 0 and out.yOmegaRB[0] == 0 and out.zOmegaRB[0] == 0


@pytest.mark.parametrize("fp64", [False, True])
def test_oracle_rigid_free_fall(fp64):
    p = dam_params(0.02, 1e-3)
    check_free_fall(OracleBackend(p, fp64=fp64), p, lone_cube(p))


def test_oracle_fp32_rigid_coupling_against_fp64():
    """Three coupled steps of the floating-cubes scene: FP32 vs FP64 oracle. Measured
    differences are ~1e-5 relative on body velocities; bounds below leave 10-100x margin."""
    st, dmin, dmax, p = S.floating_cubes()
    outs = []
    for fp64 in (False, True):
        o = OracleBackend(p, fp64=fp64)
        o.set_sim_domain_bounds(dmin, dmax)
        o.pull(st, p)
        o.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
        for _ in range(3):
            o.step(p)
        outs.append(o.push())
    a, b = outs
    for n, tol in (("yCM", 1e-6), ("xVelRB", 1e-3), ("yVelRB", 1e-3), ("zVelRB", 1e-3), ("xOmegaRB", 2e-3),
                   ("yOmegaRB", 2e-3), ("zOmegaRB", 2e-3)):
        x, y = getattr(a, n).astype(np.float64), getattr(b, n).astype(np.float64)
        assert np.all(np.abs(x - y) <= tol * (np.abs(y) + np.max(np.abs(y)))), n


# ---- rigid contact solver (SolveRigidContacts, rigid_solver.cpp:602-799)
def pressed_pair(p, gap=-0.010, edge=0.16):
    """Two hollow cubes (densities 800 and 1200 kg/m^3) overlapping by -gap along x in free space:
    no fluid, no walls; gravity is switched off by the caller."""
    boxes = [S.OBB((1.0, 1.0, 1.0), (edge, edge, edge)), S.OBB((1.0 + edge + gap, 1.0, 1.0), (edge, edge, edge))]
    parts = [S.rigid_hollow_box(b, p, d) for b, d in zip(boxes, (800.0, 1200.0))]
    nr = sum(loc[0].shape[0] for loc, _ in parts)
    st = S.UniversalSimState(0, 0, nr, 2, p.restDensity)
    at = 0
    for k, (loc, body) in enumerate(parts):
        n = loc[0].shape[0]
        st.xPosRelR[at:at + n], st.yPosRelR[at:at + n], st.zPosRelR[at:at + n] = loc
        st.bodyIdR[at:at + n] = k
        at += n
        st.xCM[k], st.yCM[k], st.zCM[k] = body["center"]
        st.massRB[k], st.massInvRB[k] = body["mass"], body["massInv"]
        st.iBodyInv00[k], st.iBodyInv11[k], st.iBodyInv22[k] = body["iBodyInv"]
        for r in range(3):
            for c in range(3):
                getattr(st, f"a{r}{c}")[k] = body["A"][r, c]
        st.rigidParticleCountRB[k] = n
    st.psiR[:] = p.massB
    st.volR[:] = np.float32(p.massB / p.restDensity)
    return st


def run_pair(be, p, st, steps=4):
    be.pull(st, p)
    be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    reports = []
    for _ in range(steps):
        be.step(p)
        reports.append(be.contact_report())
    return be.push(), reports


def test_oracle_contact_idle_without_contact():
    p = dam_params(0.02, 1e-3)
    o = OracleBackend(p)
    o.pull(lone_cube(p), p)
    o.step(p)
    r = o.contact_report()
    assert r.solverIters == 0 and r.converged == 1 and r.nContacts == 0 and r.nContactBoundary == 0


@pytest.mark.parametrize("fp64", [False, True])
def test_oracle_contact_conserves_momentum_and_separates(fp64):
    """Contact forces between two bodies are equal and opposite (f_ij = -f_ji in the SPH contact
    pressure force), so two overlapping cubes at rest in free space gain opposite momenta and
    move apart."""
    p = dam_params(0.02, 1e-3)
    p.gravity = (0.0, 0.0, 0.0)
    st = pressed_pair(p)
    out, reports = run_pair(OracleBackend(p, fp64=fp64), p, st)
    assert any(r.solverIters > 0 for r in reports)
    m = st.massRB.astype(np.float64)
    px = float(np.sum(m * out.xVelRB))
    scale = float(np.max(np.abs(m * out.xVelRB)))
    assert scale > 0
    assert abs(px) <= 1e-5 * scale
    assert out.xVelRB[0] < 0.0 < out.xVelRB[1]


def test_oracle_fp32_contact_against_fp64():
    """Stacked cubes pressed into the floor and each other: FP32 vs FP64 oracle body states after
    four steps; the contact iteration counts agree."""
    st, dmin, dmax, p = S.stacked_cubes()
    outs, reps = [], []
    for fp64 in (False, True):
        o = OracleBackend(p, fp64=fp64)
        o.set_sim_domain_bounds(dmin, dmax)
        o.pull(st, p)
        o.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
        r = []
        for _ in range(4):
            o.step(p)
            r.append(o.contact_report().solverIters)
        outs.append(o.push())
        reps.append(r)
    assert max(reps[0]) > 0
    assert all(abs(a - b) <= 1 for a, b in zip(*reps))
    a, b = outs
    for n, tol in (("yCM", 1e-4), ("xVelRB", 2e-2), ("yVelRB", 2e-2), ("zOmegaRB", 2e-2)):
        x, y = getattr(a, n).astype(np.float64), getattr(b, n).astype(np.float64)
        assert np.all(np.abs(x - y) <= tol * (np.abs(y) + np.max(np.abs(y)))), n
