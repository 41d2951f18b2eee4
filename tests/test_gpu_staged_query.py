"""The count pass with the neighboring cell blocks staged in shared memory
(`KQueryFluidCountStaged`: one TMA bulk copy per cell of the block's stencil box, then the walks
read shared memory), pinned through the autotuner's table at every size class.

Every neighbor structure must be bit-exact with the oracle, and the state after steps
bit-identical to the plain count pass: uniform and clustered points (blocks that fit the stage
and blocks that fall back to global memory), the reference's small-cell scenes (reach 2 and 4,
whose boxes exceed the stage), the 32K dam, and a served batch (blocks spanning two scenes fall
back)."""
import numpy as np
import pytest

import kat_cases as K
from oracle import OracleBackend
from parity_util import assert_neighbor_structures_equal
from test_gpu_batch import BUDGET, assert_same_state, small_dam
from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import ServedBatchB200, SimBackendB200

pytestmark = pytest.mark.gpu

STAGED = [dict(slots=1, min_blocks=4), dict(slots=1, min_blocks=5)]
PLAIN = dict(slots=0, min_blocks=9)


def pin_count(cfg):
    """Pins the count pass to one configuration for every particle count."""
    abi.reset_tuning()
    abi.pin_tuning({f"KQueryFluidCount/n{1 << k}": cfg for k in range(22)})


@pytest.fixture(autouse=True)
def fresh_tuning():
    abi.reset_tuning()
    yield
    abi.reset_tuning()


@pytest.mark.parametrize("cfg", STAGED, ids=lambda c: f"mb{c['min_blocks']}")
@pytest.mark.parametrize("dist,n", [("uniform", 50_000), ("clustered", 50_000), ("uniform", 1 << 20)])
def test_staged_count_pass_bit_exact(dist, n, cfg):
    pin_count(cfg)
    st, dmin, dmax, p = S.neighbor_search_scene(n, dist, seed=11)
    g, o = SimBackendB200(p), OracleBackend(p)
    for be in (g, o):
        be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)
        be.neighbor_search(p)
    assert_neighbor_structures_equal(g, o, st.N_F, 0, 0, what=f"staged {dist} {n}")


REF_CASES = [(n, 1.0) for n in K.NS_SCENES] + [("small_cells", 0.5), ("small_cells", 0.25)]


def test_staged_count_pass_reference_scenes():
    """tests/unit/neighbor_search.cpp scenes with fluid, boundary and rigid particles."""
    pin_count(STAGED[0])
    for name, ratio in REF_CASES:
        p = K.ns_params(ratio)
        scene = K.NS_SCENES[name]
        st = K.make_particles(**scene)
        g, o = SimBackendB200(p), OracleBackend(p)
        for be in (g, o):
            be.pull(st, p)
            be.neighbor_search(p)
        assert K.backend_neighbors(g, g.push()) == K.reference_neighbors(scene, 1.0), name
        assert_neighbor_structures_equal(g, o, st.N_F, st.N_B, st.N_R, what=name)


def test_staged_count_pass_dam_steps_identical_to_plain():
    out = []
    for cfg in (PLAIN, STAGED[0]):
        pin_count(cfg)
        st, dmin, dmax, p = S.dam_32k()
        g = SimBackendB200(p)
        g.set_sim_domain_bounds(dmin, dmax)
        g.pull(st, p)
        g.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
        g.step(p, 20)
        out.append(g.push())
        if cfg is STAGED[0]:
            o = OracleBackend(p)
            o.set_sim_domain_bounds(dmin, dmax)
            o.pull(out[-1], p)
            o.neighbor_search(p)
            g.neighbor_search(p)
            assert_neighbor_structures_equal(g, o, st.N_F, st.N_B, st.N_R, what="dam after 20 steps")
        g.close()
    assert_same_state(out[1], out[0], exact=True, what="staged vs plain count pass")


def test_staged_count_pass_served_batch_identical_to_plain():
    scenes = [small_dam(n, 20 + n) for n in (9, 14, 11)]
    p = scenes[0][3]
    res = []
    for cfg in (PLAIN, STAGED[1]):
        pin_count(cfg)
        b = ServedBatchB200(p, BUDGET)
        slots = [b.admit(st, dmin, dmax) for st, dmin, dmax, _ in scenes]
        b.substep(3)
        res.append([(b.push(s), b.stats(s).solverIters) for s in slots])
        b.close()
    for k, ((a, ia), (c, ic)) in enumerate(zip(res[0], res[1])):
        assert ia == ic, k
        assert_same_state(c, a, exact=True, what=f"scene {k}")
