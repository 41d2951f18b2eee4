"""Served batch (`tsp_b200_batch_*`): scenes advanced together over one scene-offset fluid
array give the results they give alone.

- one scene in a batch vs the one-scene backend: same particle order (bit-exact sort), same
  Jacobi iteration counts, fields equal to FP32 round-off (the only difference is the order of
  the FP64 residual sums that decide convergence);
- a scene alone in a batch vs the same scene among other scenes of different sizes, admitted
  and retired at different substeps: bit-identical state.
"""
import numpy as np
import pytest

from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import ServedBatchB200, SimBackendB200, TspError

pytestmark = pytest.mark.gpu

BUDGET = 8 << 30


def small_dam(n_side, seed):
    """n_side^3 dam in a tank twice the block per axis, with boundary volumes computed once."""
    spec = S.ServedSceneSpec(0, n_side, n_side + 2, n_side - 1, 0.02, 1e-3, 0.0, seed)
    st, dmin, dmax, p = spec.build()
    be = SimBackendB200(p)
    be.set_sim_domain_bounds(dmin, dmax)
    be.pull(st, p)
    be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    st = be.push()
    be.close()
    return st, dmin, dmax, p


def assert_same_state(a, b, exact=True, what=""):
    assert np.array_equal(a.idF, b.idF), f"{what}: fluid order"
    for n in ("xPosF", "yPosF", "zPosF", "xVelF", "yVelF", "zVelF", "pressureF", "densityF"):
        x, y = getattr(a, n), getattr(b, n)
        if exact:
            assert np.array_equal(x, y), f"{what}: {n}"
        else:
            scale = np.max(np.abs(y)) + 1e-30
            assert np.max(np.abs(x - y)) <= 1e-5 * scale, f"{what}: {n}"


def test_batch_scene_matches_one_scene_backend():
    st, dmin, dmax, p = small_dam(14, 3)
    one = SimBackendB200(p)
    one.set_sim_domain_bounds(dmin, dmax)
    one.pull(st, p)
    bat = ServedBatchB200(p, BUDGET)
    slot = bat.admit(st, dmin, dmax)
    for k in range(4):
        one.step(p)
        bat.substep(1)
        assert bat.stats(slot).solverIters == one.stats().solverIters, f"step {k}"
    assert_same_state(bat.push(slot), one.push(), exact=False, what="batch vs one-scene backend")


def test_batch_results_do_not_depend_on_the_mix():
    scenes = [small_dam(n, 10 + n) for n in (9, 14, 11)]
    alone = []
    for st, dmin, dmax, p in scenes:
        b = ServedBatchB200(p, BUDGET)
        slot = b.admit(st, dmin, dmax)
        b.substep(3)
        alone.append((b.push(slot), b.stats(slot).solverIters))
        b.close()
    p = scenes[0][3]
    mix = ServedBatchB200(p, BUDGET)
    slots = [mix.admit(st, dmin, dmax) for st, dmin, dmax, _ in scenes]
    mix.substep(3)
    for k, slot in enumerate(slots):
        assert mix.stats(slot).solverIters == alone[k][1]
        assert_same_state(mix.push(slot), alone[k][0], exact=True, what=f"scene {k} in the mix")


def test_batch_continuous_admission_and_retirement():
    """Scene B joins after two substeps of scene A, A retires after two more; B's state after
    three substeps equals B run alone for three substeps."""
    (sa, da0, da1, p), (sb, db0, db1, _) = small_dam(12, 21), small_dam(10, 22)
    ref = ServedBatchB200(p, BUDGET)
    rb = ref.admit(sb, db0, db1)
    ref.substep(3)
    want = ref.push(rb)
    ref.close()
    bat = ServedBatchB200(p, BUDGET)
    a = bat.admit(sa, da0, da1)
    bat.substep(2)
    b = bat.admit(sb, db0, db1)
    bat.substep(2)
    out_a = bat.retire(a, push=True)
    assert out_a.step == 4
    bat.substep(1)
    got = bat.push(b)
    assert got.step == 3
    assert_same_state(got, want, exact=True, what="scene admitted mid-stream")
    assert bat.info()["scenes"] == 1


def test_batch_refuses_scene_over_budget():
    st, dmin, dmax, p = small_dam(9, 5)
    bat = ServedBatchB200(p, 1 << 20)
    with pytest.raises(TspError) as e:
        bat.admit(st, dmin, dmax)
    assert e.value.status == -3


def test_batch_scenes_match_oracle():
    """Each scene of a mix against the oracle (the reference CPU step restated) stepping that
    scene alone: same particle order (bit-exact sort), same Jacobi iteration counts, fields within
    the full-step bounds of the one-scene parity test (the GPU's hardware reciprocal square root
    and FP64 sum order are the differences; bounds grow with the step)."""
    from oracle import OracleBackend
    from parity_util import assert_elementwise
    scenes = [small_dam(n, 30 + n) for n in (9, 12, 10)]
    mix = ServedBatchB200(scenes[0][3], BUDGET)
    slots = [mix.admit(st, dmin, dmax) for st, dmin, dmax, _ in scenes]
    oracles = []
    for st, dmin, dmax, p in scenes:
        o = OracleBackend(p)
        o.set_sim_domain_bounds(dmin, dmax)
        o.pull(st, p)
        oracles.append(o)
    for k in range(3):
        mix.substep(1)
        s1 = k + 1
        for slot, o, (_, _, _, p) in zip(slots, oracles, scenes):
            o.step(p)
            assert mix.stats(slot).solverIters == o.stats().solverIters, (k, slot)
            gs, os_ = mix.push(slot), o.push()
            assert np.array_equal(gs.idF, os_.idF), (k, slot)
            for name, rtol, atol, frac in (("densityF", 1e-5 * s1, 1e-2 * s1, 0.0),
                                           ("pressureF", 1e-3 * s1, 1.0 * s1, 0.0),
                                           ("xPosF", 1e-6, 1e-7 * s1, 0.0), ("yVelF", 1e-3 * s1, 1e-5 * s1, 0.0),
                                           ("xAccPressF", 1e-3 * s1, 0.0, 1e-4 * s1),
                                           ("sourceTermF", 1e-3 * s1, 1e-2 * s1, 0.0),
                                           ("diagElemF", 1e-4 * s1, 0.0, 1e-5 * s1)):
                ref = getattr(os_, name)
                assert_elementwise(getattr(gs, name), ref, rtol, atol + frac * float(np.abs(ref).max()),
                                   f"substep {k} slot {slot} {name}")
