"""Export and resume through TSPSIM2 state files on the GPU backend.

A run pushed to the host, written to a state file, loaded and pulled into a fresh backend
continues like the run that never stopped:
- fluid-only dam (32K): bit-identical positions, velocities, pressures and densities after 8 more
  steps -- every fluid and boundary field the step reads is in the file, and the push order is
  the backend's own particle order, so the resumed sort sees the same keys in the same order;
- floating cubes: the body state lives in FP64 on the device and the file holds FP32 (as the
  reference's state does), so the resumed run agrees within 1e-5 m in the centres of mass and
  1e-4 m/s in the body and fluid velocities after 8 more steps.
"""
import numpy as np
import pytest

from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import SimBackendB200
from turbospharticles_b200.state_io import load_universal_sim_state, save_universal_sim_state

pytestmark = pytest.mark.gpu

FLUID = ["idF", "xPosF", "yPosF", "zPosF", "xVelF", "yVelF", "zVelF", "pressureF", "densityF"]


def started(builder, steps):
    st, dmin, dmax, p = builder()
    g = SimBackendB200(p)
    g.set_sim_domain_bounds(dmin, dmax)
    g.pull(st, p)
    g.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    for _ in range(steps):
        g.step(p)
    return g, p, dmin, dmax


def resumed(path, p, dmin, dmax):
    st = load_universal_sim_state(path)
    r = SimBackendB200(p)
    r.set_sim_domain_bounds(dmin, dmax)
    r.pull(st, p)
    return r, st


def test_gpu_fluid_resume_is_bit_identical(tmp_path):
    g, p, dmin, dmax = started(S.dam_32k, 5)
    saved = g.push()
    path = str(tmp_path / "state.bin")
    save_universal_sim_state(saved, path)
    r, st = resumed(path, p, dmin, dmax)
    assert (st.step, st.time) == (saved.step, saved.time)
    for _ in range(8):
        g.step(p)
        r.step(p)
    a, b = g.push(), r.push()
    assert (a.step, a.time) == (b.step, b.time)
    for n in FLUID:
        np.testing.assert_array_equal(getattr(a, n), getattr(b, n), n)


def test_gpu_rigid_resume_within_bounds(tmp_path):
    g, p, dmin, dmax = started(S.floating_cubes, 5)
    path = str(tmp_path / "state.bin")
    save_universal_sim_state(g.push(), path)
    r, st = resumed(path, p, dmin, dmax)
    assert st.N_RB > 0 and st.N_R > 0
    for _ in range(8):
        g.step(p)
        r.step(p)
    a, b = g.push(), r.push()
    np.testing.assert_array_equal(a.idR, b.idR)
    for c in ("xCM", "yCM", "zCM"):
        assert np.max(np.abs(getattr(a, c).astype(np.float64) - getattr(b, c))) <= 1e-5, c
    for c in ("xVelRB", "yVelRB", "zVelRB"):
        assert np.max(np.abs(getattr(a, c).astype(np.float64) - getattr(b, c))) <= 1e-4, c
    ia, ib = np.argsort(a.idF), np.argsort(b.idF)
    for c in ("xVelF", "yVelF", "zVelF"):
        assert np.max(np.abs(getattr(a, c)[ia].astype(np.float64) - getattr(b, c)[ib])) <= 1e-4, c
