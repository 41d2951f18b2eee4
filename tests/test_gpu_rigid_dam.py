"""Rigid coupling at full size: the double dam break with 2,000,000 fluid particles
(two 100 x 125 x 80 blocks, dx = 0.008 m, 4 x 1.5 x 1.5 m tank) and 8 hollow cubes of edge
0.15 m (3,088 boundary particles each; 4 at 500 kg/m^3, 4 at 2,000 kg/m^3) with seeded
orientations, dropped at 1 m/s onto the two blocks' top faces, so that fluid-rigid forces and
torques act from the first step.

- Rigid trajectories against the FP64 oracle over a prefix of PREFIX_STEPS coupled steps (the
  GPU computes per-particle terms in FP32, body sums and the body integrator in FP64): centres
  of mass within CM_ATOL, body velocities and angular velocities within VEL_RTOL of the largest
  body speed (angular: of the largest angular speed), identical Jacobi iteration counts.
- Then LONG_STEPS further GPU steps with bounds: every centre of mass inside the tank, all
  body and fluid states finite, the average positive density error at most the solver target
  whenever the solver stopped before its iteration limit.
"""
import numpy as np
import pytest

from oracle import OracleBackend
from parity_util import report
from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import SimBackendB200

pytestmark = pytest.mark.gpu

PREFIX_STEPS = 20
LONG_STEPS = 480
CM_ATOL = 1e-5
VEL_RTOL = 2e-3


def _body(s):
    cm = np.stack([s.xCM, s.yCM, s.zCM], 1).astype(np.float64)
    v = np.stack([s.xVelRB, s.yVelRB, s.zVelRB], 1).astype(np.float64)
    w = np.stack([s.xOmegaRB, s.yOmegaRB, s.zOmegaRB], 1).astype(np.float64)
    return cm, v, w


def test_gpu_rigid_dam_full_size():
    st, dmin, dmax, p = S.rigid_dam()
    assert (st.N_F, st.N_RB, st.N_R) == (2_000_000, 8, 8 * 3088)
    g, d = SimBackendB200(p), OracleBackend(p, fp64=True)
    for be in (g, d):
        be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)
        be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    rows = []
    for k in range(1, PREFIX_STEPS + 1):
        g.step(p)
        d.step(p)
        assert g.stats().solverIters == d.stats().solverIters, k
        (cg, vg, wg), (cd, vd, wd) = _body(g.push()), _body(d.push())
        vs = max(float(np.abs(vd).max()), 1e-6)
        ws = max(float(np.abs(wd).max()), 1e-6)
        rows.append(dict(step=k, cm_err=float(np.abs(cg - cd).max()), vel_err=float(np.abs(vg - vd).max()),
                         vel_scale=vs, omega_err=float(np.abs(wg - wd).max()), omega_scale=ws))
    report("rigid_dam_prefix", rows)
    for r in rows:
        assert r["cm_err"] <= CM_ATOL, r
        assert r["vel_err"] <= VEL_RTOL * r["vel_scale"], r
        assert r["omega_err"] <= VEL_RTOL * r["omega_scale"], r
    del d
    lo = np.asarray(dmin, np.float64) - 0.05
    hi = np.asarray(dmax, np.float64) + 0.05
    target = float(np.float32(p.densityDevTarget))
    for k in range(LONG_STEPS):
        g.step(p)
        sg = g.stats()
        if sg.solverIters < p.maxSolverIters:
            assert sg.avgRelDensityErrPos <= target, (k, sg.avgRelDensityErrPos)
    s = g.push()
    cm, v, w = _body(s)
    assert np.all(np.isfinite(cm)) and np.all(np.isfinite(v)) and np.all(np.isfinite(w))
    assert np.all(cm >= lo) and np.all(cm <= hi), cm
    assert np.all(np.isfinite(s.xPosF)) and np.all(np.isfinite(s.yVelF))
    report("rigid_dam_long", dict(steps=PREFIX_STEPS + LONG_STEPS, cm=cm.tolist(), vel=v.tolist()))
