"""Pins the CPU oracle to the known answers of the reference's own unit tests (no GPU)."""
import math

import numpy as np
import pytest

import kat_cases as K
from oracle import OracleBackend, kernel_eval
from turbospharticles_b200 import abi

f32 = np.float32


@pytest.mark.parametrize("i,dist,weight,grad", [
    (0, 0.0, 1.0, 0.0), (1, 0.5, 23 / 32, -15 / 16), (2, 1.0, 0.25, -0.75),
    (3, 1.5, 1 / 32, -3 / 16), (4, 2.0, 0.0, 0.0), (5, 2.5, 0.0, 0.0)])
def test_kernel_known_values(i, dist, weight, grad):
    """tests/unit/sph_kernels.cpp:116-144 (h = 1, alpha = 1 / (4 pi))."""
    w, kg, gx, gy, gz = kernel_eval(dist, 0.0, 0.0, 1.0, 4.0, K.alpha_of(1.0))
    assert abs(w - weight / math.pi) <= 1e-7
    assert abs(gx - grad / math.pi) <= 1e-7
    assert gy == 0.0 and gz == 0.0


@pytest.mark.parametrize("h", [0.25, 0.7, 1.0, 4.0])
def test_kernel_matches_closed_form(h):
    """tests/unit/sph_kernels.cpp:146-167 (tolerance 1e-7 + 2e-6 |x| on dimensionless values)."""
    offsets = [(0.125, -0.25, 0.375), (-0.5, 0.25, -0.125), (0.0, 0.6, -0.8), (0.75, -1.0, 0.5),
               (-1.0, 0.5, 1.25), (1.5, 1.5, 0.25), (0.3, -0.4, 0.25), (0.9, -1.2, 0.0)]
    hf = float(f32(h))
    size_inv = float(f32(1.0 / hf))
    for o in offsets:
        off = (np.array(o, f32) * f32(h)).astype(f32)
        w, kg, gx, gy, gz = kernel_eval(*[float(v) for v in off], size_inv, float(f32(4 * h * h)), K.alpha_of(h))
        rw, rg = K.kernel_reference(off.astype(np.float64), hf)
        ws, gs = hf ** 3, hf ** 4
        assert abs(w * ws - rw * ws) <= 1e-7 + 2e-6 * abs(rw * ws)
        # the SIMD gradient uses the no-min-distance factor times the offset
        g = np.array([kg * float(off[0]), kg * float(off[1]), kg * float(off[2])])
        for a in range(3):
            assert abs(g[a] * gs - rg[a] * gs) <= 1e-7 + 2e-6 * abs(rg[a] * gs)


def test_pressure_pair_known_answers():
    """tests/unit/sph_pressure.cpp:391-463 on the oracle."""
    o = OracleBackend(K.pressure_params())
    K.check_pressure_pair(K.pressure_pair_kats(o))


def test_density_known_fluid_contribution():
    st, p, expected = K.density_kat_state()
    o = OracleBackend(p)
    o.pull(st, p)
    o.neighbor_search(p)
    o.run_stage(abi.STAGE_DENSITY, p)
    ids = o.push().idF
    d = o.read_field(abi.FIELD_DENSITY)
    first = int(np.where(ids == 0)[0][0])
    assert abs(d[first] - expected) <= 1e-7 + 3e-6 * abs(expected)


@pytest.mark.parametrize("mass,rho_j", [(1.0, 2.0), (1.0, 5.0), (3.0, 2.0), (3.0, 5.0)])
def test_fluid_viscosity_known_answer(mass, rho_j):
    st, p, expected = K.viscosity_kat_state(mass, rho_j)
    o = OracleBackend(p)
    o.pull(st, p)
    o.neighbor_search(p)
    o.run_stage(abi.STAGE_NON_PRESSURE, p)
    ids = o.push().idF
    vp = o.read_field(abi.FIELD_VEL_PRED)
    first = int(np.where(ids == 0)[0][0])
    assert abs(vp[first, 0] - expected) <= 2e-6 + 8e-6 * abs(expected)
    assert vp[first, 1] == 2.0 and vp[first, 2] == 3.0


@pytest.mark.parametrize("case", range(4))
def test_integration_exact(case):
    (x, vp, a), dt, (x1, v1) = K.integration_kats()[case]
    p = K.SimParams(timeStep=dt)
    st = K.UniversalSimState(1, 0, 0, 0)
    st.xPosF[:], st.yPosF[:], st.zPosF[:] = x
    st.xVelPredF[:], st.yVelPredF[:], st.zVelPredF[:] = vp
    st.xAccPressF[:], st.yAccPressF[:], st.zAccPressF[:] = a
    st.xVelF[:] = 100.0
    o = OracleBackend(p)
    o.pull(st, p)
    o.run_stage(abi.STAGE_INTEGRATION, p)
    assert np.array_equal(o.read_field(abi.FIELD_POS)[0], np.array(x1, np.float64))
    assert np.array_equal(o.read_field(abi.FIELD_VEL)[0], np.array(v1, np.float64))


def _ns_case_ids():
    cases = [(name, 1.0) for name in K.NS_SCENES]
    cases += [("small_cells", r) for r in (0.5, 0.25)]
    cases += [(f"simd_{n}", 1.0) for n in (15, 16, 17, 31, 32, 33)]
    cases += [(f"dense_{n}", 1.0) for n in (256, 272)]
    return cases


def ns_scene(name):
    if name.startswith("simd_"):
        return K.simd_width_scene(int(name.split("_")[1]))
    if name.startswith("dense_"):
        return K.dense_lattice_scene(int(name.split("_")[1]))
    return K.NS_SCENES[name]


@pytest.mark.parametrize("name,ratio", _ns_case_ids())
def test_oracle_neighbor_sets_match_fp64_all_pairs(name, ratio):
    """tests/unit/neighbor_search.cpp:139-177 on the oracle: sorted neighbor-ID lists per
    category equal the FP64 all-pairs reference."""
    scene = ns_scene(name)
    p = K.ns_params(ratio)
    o = OracleBackend(p)
    o.pull(K.make_particles(**scene), p)
    o.neighbor_search(p)
    got = K.backend_neighbors(o, o.push())
    assert got == K.reference_neighbors(scene, 1.0)


def test_oracle_rows_ascending_and_self_included():
    scene = K.dense_lattice_scene(272)
    p = K.ns_params()
    o = OracleBackend(p)
    o.pull(K.make_particles(**scene), p)
    o.neighbor_search(p)
    for lst in range(6):
        off, idx = o.rows(lst)
        for i in range(len(off) - 1):
            row = idx[off[i]:off[i + 1]]
            assert np.all(np.diff(row.astype(np.int64)) > 0)
            if lst == 0:
                assert i in set(row.tolist())


def test_oracle_sell32_roundtrip():
    """The SELL32 encoding of the oracle rows decodes back to the rows (both formats)."""
    from turbospharticles_b200 import scene as S
    st, dmin, dmax, p = S.neighbor_search_scene(20000, "clustered", seed=3)
    o = OracleBackend(p)
    o.set_sim_domain_bounds(dmin, dmax)
    o.pull(st, p)
    o.neighbor_search(p)
    for lst in range(3):
        off, idx = o.rows(lst)
        m = o.sell32(lst)
        n = st.N_F
        for i in range(0, n, 97):
            c, lane = divmod(i, 32)
            row = []
            for k in range(int(m["counts"][i])):
                lin = int(m["offset"][c]) + k * 32 + lane
                if m["format"][c] == 0:
                    e = int(m["w16"][lin])
                    row.append(int(m["base2"][c]) + (e & 0x7FFF) if e & 0x8000 else int(m["base"][c]) + e)
                else:
                    row.append(int(m["w32"][lin]))
            assert row == idx[off[i]:off[i + 1]].tolist()
