"""Parity of the B200 backend with the CPU oracle and the reference's known answers.

Neighbor structures (Morton cell IDs, sort permutation, cell tables, neighbor rows, SELL32
chunk metadata and packed words) must be bit-exact. FP32 solver fields compare element by
element, |gpu - oracle| <= rtol * |oracle| + atol, rtol and the absolute floor atol stated per
field by each test.
"""
import numpy as np
import pytest

import kat_cases as K
from oracle import OracleBackend
from parity_util import assert_elementwise, assert_neighbor_structures_equal
from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import SimBackendB200

pytestmark = pytest.mark.gpu


def pair(p, fp64=False):
    return SimBackendB200(p), OracleBackend(p, fp64=fp64)


def load(bes, st, p, dmin=None, dmax=None):
    for be in bes:
        if dmin is not None:
            be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)


# ------------------------------------------------------------------------------ known answers
def test_gpu_pressure_pair_known_answers():
    K.check_pressure_pair(K.pressure_pair_kats(SimBackendB200(K.pressure_params())))


def test_gpu_density_and_viscosity_known_answers():
    st, p, expected = K.density_kat_state()
    g = SimBackendB200(p)
    g.pull(st, p)
    g.neighbor_search(p)
    g.run_stage(abi.STAGE_DENSITY, p)
    ids = g.push().idF
    d = g.read_field(abi.FIELD_DENSITY)
    assert abs(d[int(np.where(ids == 0)[0][0])] - expected) <= 1e-7 + 3e-6 * abs(expected)
    for mass, rho in ((1.0, 2.0), (3.0, 5.0)):
        st, p, expected = K.viscosity_kat_state(mass, rho)
        g = SimBackendB200(p)
        g.pull(st, p)
        g.neighbor_search(p)
        g.run_stage(abi.STAGE_NON_PRESSURE, p)
        ids = g.push().idF
        vp = g.read_field(abi.FIELD_VEL_PRED)
        k = int(np.where(ids == 0)[0][0])
        assert abs(vp[k, 0] - expected) <= 2e-6 + 8e-6 * abs(expected)


def test_gpu_integration_exact():
    for (x, vp, a), dt, (x1, v1) in K.integration_kats():
        p = K.SimParams(timeStep=dt)
        st = K.UniversalSimState(1, 0, 0, 0)
        st.xPosF[:], st.yPosF[:], st.zPosF[:] = x
        st.xVelPredF[:], st.yVelPredF[:], st.zVelPredF[:] = vp
        st.xAccPressF[:], st.yAccPressF[:], st.zAccPressF[:] = a
        g = SimBackendB200(p)
        g.pull(st, p)
        g.run_stage(abi.STAGE_INTEGRATION, p)
        assert np.array_equal(g.read_field(abi.FIELD_POS)[0], np.array(x1, np.float32))
        assert np.array_equal(g.read_field(abi.FIELD_VEL)[0], np.array(v1, np.float32))


# ------------------------------------------------------------------------------ neighbor search
NS_CASES = [(n, 1.0) for n in K.NS_SCENES] + [("small_cells", 0.5), ("small_cells", 0.25)] + \
    [(f"simd_{n}", 1.0) for n in (15, 16, 17, 31, 32, 33, 63, 65)] + [(f"dense_{n}", 1.0) for n in (256, 272)]


def ns_scene(name):
    if name.startswith("simd_"):
        return K.simd_width_scene(int(name.split("_")[1]))
    if name.startswith("dense_"):
        return K.dense_lattice_scene(int(name.split("_")[1]))
    return K.NS_SCENES[name]


@pytest.mark.parametrize("name,ratio", NS_CASES)
def test_gpu_reference_neighbor_scenes(name, ratio):
    """tests/unit/neighbor_search.cpp scenes: FP64 all-pairs sets, and bit-exact structures."""
    scene = ns_scene(name)
    p = K.ns_params(ratio)
    st = K.make_particles(**scene)
    g, o = pair(p)
    load((g, o), st, p)
    g.neighbor_search(p)
    o.neighbor_search(p)
    assert K.backend_neighbors(g, g.push()) == K.reference_neighbors(scene, 1.0)
    assert_neighbor_structures_equal(g, o, st.N_F, st.N_B, st.N_R)


def test_gpu_search_after_particles_move():
    """neighbor_search.cpp:347-371: repeated imports of moved scenes reuse the backend."""
    orig = dict(fluid=[(0, 0, 0), (0.5, 0, 0), (-4, 0.25, 0.25)], boundary=[(0.25, 0, 0), (-4.25, 0.25, 0.25)],
                rigid=[(0.75, 0, 0), (-4, 0.5, 0.25)])
    moved = dict(fluid=[(32, 0, 0), (-4.5, 0.25, 0.25), (-4, 0.25, 0.25)],
                 boundary=[(32.25, 0, 0), (-4.25, 0.25, 0.25)], rigid=[(32.75, 0, 0), (-4, 0.5, 0.25)])
    shifted = {k: [tuple(np.add(v, (64, -16, 8))) for v in vs] for k, vs in moved.items()}
    p = K.ns_params()
    g = SimBackendB200(p)
    for sc in (orig, moved, shifted, orig):
        g.pull(K.make_particles(**sc), p)
        g.neighbor_search(p)
        assert K.backend_neighbors(g, g.push()) == K.reference_neighbors(sc, 1.0)


@pytest.mark.parametrize("dist,n", [("uniform", 50_000), ("clustered", 50_000), ("uniform", 1 << 20),
                                    ("clustered", 1 << 20), ("uniform", 1 << 22), ("clustered", 1 << 22)])
def test_gpu_neighbor_search_bit_exact(dist, n):
    """Neighbor-search workload at its two sizes, 1,048,576 and 4,194,304 points (uniform /
    16 Gaussian blobs + 20 % background in the unit cube, ~50 neighbors for uniform; the
    clustered 4M rows reach ~1,900 entries, with Abs32 and home/far split chunks): every
    structure bit-exact with the oracle."""
    st, dmin, dmax, p = S.neighbor_search_scene(n, dist, seed=7)
    g, o = pair(p)
    load((g, o), st, p, dmin, dmax)
    g.neighbor_search(p)
    o.neighbor_search(p)
    assert_neighbor_structures_equal(g, o, st.N_F, 0, 0)


def test_gpu_neighbor_lists_grow_between_builds():
    """A build whose lists outgrow the buffers sized by the previous build (a sparse first
    scene keeps them small): the buffers grow in place and the structures are still bit-exact
    with the oracle."""
    st, dmin, dmax, p = S.neighbor_search_scene(1 << 20, "uniform", seed=7)
    sparse = st.copy()
    for c in ("xPosF", "yPosF", "zPosF"):
        setattr(sparse, c, (getattr(st, c) * np.float32(3.0)).astype(np.float32))
    g, o = pair(p)
    g.set_sim_domain_bounds(np.asarray(dmin, np.float32) * 3, np.asarray(dmax, np.float32) * 3)
    g.pull(sparse, p)
    g.neighbor_search(p)
    load((g, o), st, p, dmin, dmax)
    g.neighbor_search(p)
    o.neighbor_search(p)
    assert_neighbor_structures_equal(g, o, st.N_F, 0, 0)


def test_gpu_neighbor_search_particles_outside_the_frame():
    """Points over [0, 2]^3 with the unit cube as simulation domain: the frame is the bounds
    clamped to the domain and widened by reach + 8 cells (neighbor_search.cpp:1902-2005), so
    about half the points lie beyond it. They get the empty cell ID, sort last (stable) and
    have no rows; every structure bit-exact with the oracle."""
    st, dmin, dmax, p = S.neighbor_search_scene(50_000, "uniform", seed=13)
    for a in (st.xPosF, st.yPosF, st.zPosF):
        a *= np.float32(2.0)
    g, o = pair(p)
    load((g, o), st, p, dmin, dmax)
    g.neighbor_search(p)
    o.neighbor_search(p)
    cid = g.cell_ids(abi.SPECIES_F)
    empty = cid == np.uint64(0xFFFFFFFFFFFFFFFF)
    assert empty.any() and not empty.all()
    assert not empty[:int(np.argmax(empty))].any() and empty[int(np.argmax(empty)):].all(), "empty IDs sort last"
    assert_neighbor_structures_equal(g, o, st.N_F, 0, 0, what="outside the frame")
    off, _ = g.rows(abi.LIST_FF)
    assert np.all(np.diff(off.astype(np.int64))[empty] == 0)


def test_gpu_steps_without_fluid():
    """A boundary-only scene steps like the reference's empty serial simulation
    (cpu_backend.cpp:2309-2315): counters advance, no solve, the boundary is unchanged."""
    p = K.ns_params()
    st = K.make_particles(**K.NS_SCENES["boundary_only"])
    g, o = pair(p)
    load((g, o), st, p)
    for _ in range(3):
        g.step(p)
        o.step(p)
    sg, so = g.stats(), o.stats()
    assert (sg.step, sg.solverIters) == (so.step, so.solverIters) == (3, 0)
    assert sg.time == pytest.approx(so.time)
    gs, os_ = g.push(), o.push()
    assert gs.N_F == 0 and gs.N_B == os_.N_B
    order = np.argsort(gs.idB)
    assert np.array_equal(gs.xPosB[order], st.xPosB[np.argsort(st.idB)])


def test_gpu_neighbor_search_4m_properties():
    """4,194,304 uniform points, another seed than the bit-exact case: size-independent
    properties -- FF rows ascending, self included exactly for in-frame particles, the FF
    relation symmetric (checked on a seeded sample), Morton cell IDs non-decreasing."""
    st, dmin, dmax, p = S.neighbor_search_scene(1 << 22, "uniform", seed=11)
    g = SimBackendB200(p)
    g.set_sim_domain_bounds(dmin, dmax)
    g.pull(st, p)
    g.neighbor_search(p)
    off, idx = g.rows(abi.LIST_FF)
    off = off.astype(np.int64)
    n = st.N_F
    cid = g.cell_ids(abi.SPECIES_F)
    inframe = cid != np.uint64(0xFFFFFFFFFFFFFFFF)
    assert np.all(np.diff(cid[inframe].astype(np.float64)) >= 0)
    rng = np.random.default_rng(5)
    for i in rng.choice(n, 4000, replace=False):
        row = idx[off[i]:off[i + 1]].astype(np.int64)
        assert np.all(np.diff(row) > 0)
        assert (i in set(row.tolist())) == bool(inframe[i])
        for j in row[:: max(1, len(row) // 8)]:
            rj = idx[off[j]:off[j + 1]]
            k = np.searchsorted(rj, i)
            assert k < len(rj) and rj[k] == i


# ------------------------------------------------------------------------------ SPH stages
def dam_pair(fp64=False, steps_before=0):
    st, dmin, dmax, p = S.dam_32k()
    g, o = pair(p, fp64)
    load((g, o), st, p, dmin, dmax)
    for be in (g, o):
        be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    return g, o, p


def test_gpu_boundary_volumes_match_oracle():
    g, o, p = dam_pair()
    # same summation order as the reference's z-y-x cell walk; the weights' square roots are
    # IEEE on both sides, so only the compiler's operation order could differ
    gb, ob = g.push(), o.push()
    og = np.argsort(gb.idB)
    oo = np.argsort(ob.idB)
    assert_elementwise(gb.volB[og], ob.volB[oo], 1e-6, 0.0, "volB")
    assert_elementwise(gb.psiB[og], ob.psiB[oo], 1e-6, 0.0, "psiB")


def test_gpu_stages_match_oracle_from_identical_state():
    g, o, p = dam_pair()
    for be in (g, o):
        be.neighbor_search(p)
    # identical start state for every stage (fields copied from the oracle); element-wise
    # bounds rtol * |oracle| + atol with floors: density and source term 1e-3 kg/m^3, predicted
    # velocity 1e-5 g dt, pressure 1e-2 Pa; the diagonal and the pressure acceleration, sums of
    # cancelling terms, 1e-6 of their largest magnitude
    for stage, fields in (
            (abi.STAGE_DENSITY, [(abi.FIELD_DENSITY, 2e-6, 1e-3)]),
            (abi.STAGE_NON_PRESSURE, [(abi.FIELD_VEL_PRED, 2e-6, 1e-5 * 9.81 * 1e-3)]),
            (abi.STAGE_SOURCE_DIAG_INIT, [(abi.FIELD_SOURCE, 1e-4, 1e-3), (abi.FIELD_DIAG, 2e-5, None),
                                          (abi.FIELD_PRESSURE, 1e-4, 1e-2)]),
            (abi.STAGE_PRESSURE_ACC, [(abi.FIELD_ACC_PRESS, 1e-4, None)]),
            (abi.STAGE_JACOBI_UPDATE, [(abi.FIELD_PRESSURE, 1e-4, 1e-2)])):
        for f in (abi.FIELD_DENSITY, abi.FIELD_VEL_PRED, abi.FIELD_SOURCE, abi.FIELD_DIAG, abi.FIELD_PRESSURE,
                  abi.FIELD_ACC_PRESS):
            g.write_field(f, o.read_field(f))
        eg = g.run_stage(stage, p)
        eo = o.run_stage(stage, p)
        for f, rtol, atol in fields:
            ref = o.read_field(f)
            if atol is None:
                atol = 1e-6 * float(np.abs(ref).max())
            assert_elementwise(g.read_field(f), ref, rtol, atol, f"stage {stage} field {f}")
        if stage == abi.STAGE_JACOBI_UPDATE:
            # FP64 sums of per-particle FP32 terms that differ in their last bits (3.6e-9 measured)
            assert_elementwise(eg, eo, 1e-8, 0.0, "FP64 error sums")


def test_gpu_steps_match_oracle():
    """Full IISPH steps of the 32K dam from an identical start: same Jacobi iteration counts,
    fields within tolerance (FP64 sum order and the hardware reciprocal square root of the
    GPU's distances are the differences)."""
    g, o, p = dam_pair()
    for k in range(3):
        g.step(p)
        o.step(p)
        sg, so = g.stats(), o.stats()
        assert sg.solverIters == so.solverIters
        assert abs(sg.avgRelDensityErrPos - so.avgRelDensityErrPos) <= 1e-6 + 1e-3 * abs(so.avgRelDensityErrPos)
        gs, os_ = g.push(), o.push()
        assert np.array_equal(gs.idF, os_.idF), "identical particle order (bit-exact permutation)"
        # after whole steps the trajectories separate (each step starts from the previous
        # step's slightly different state): bounds grow with the step, floors as above
        s1 = k + 1
        # (field, rtol, absolute floor, floor as a fraction of the field's largest magnitude)
        for name, rtol, atol, frac in (("densityF", 1e-5 * s1, 1e-2 * s1, 0.0), ("pressureF", 1e-3 * s1, 1.0 * s1, 0.0),
                                       ("xPosF", 1e-6, 1e-7 * s1, 0.0), ("yVelF", 1e-3 * s1, 1e-5 * s1, 0.0),
                                       ("xAccPressF", 1e-3 * s1, 0.0, 1e-4 * s1),
                                       ("sourceTermF", 1e-3 * s1, 1e-2 * s1, 0.0), ("diagElemF", 1e-4 * s1, 0.0, 1e-5 * s1)):
            ref = getattr(os_, name)
            atol = atol + frac * float(np.abs(ref).max())  # cancelling sums: floor relative to the field
            assert_elementwise(getattr(gs, name), ref, rtol, atol, f"step {k} {name}")
