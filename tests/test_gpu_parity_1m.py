"""Parity on the 1,000,000-particle dam break, the workload the bench measures.

A developed state (the GPU's state after DEVELOP_STEPS steps of the collapse: non-zero
velocities, pressures and a free surface) is pulled into the GPU backend, the FP32 oracle and
the FP64 oracle. Each SPH stage then runs from an identical start (all solver fields copied
from the FP32 oracle before the stage) and its output is compared element by element:

- against the FP32 oracle within the bound stated per field below (the GPU forms distances with
  the hardware reciprocal square root and sums in the same order; the rest is FP32 rounding);
- against the FP64 oracle run on the same FP32 inputs: the FP32 error of the stage, asserted
  against the 1e-4 relative bound on per-step field error with the field's stated absolute floor.

Floors (atol): density, source term 1e-3 kg/m^3 (1e-6 of the rest density); pressure 1e-2 Pa;
predicted velocity 1e-5 g dt; the diagonal a_ii and the pressure acceleration, sums of
cancelling terms, 1e-6 of their largest magnitude in the scene. Below a floor a value is
compared in absolute terms.

Measured on a B200 (largest relative error above the floor, GPU against the FP64 oracle):
density 5.2e-7, predicted velocity 6.3e-7, source term 6.2e-7, diagonal 1.2e-6, initial
pressure 3.2e-5, pressure acceleration 9.3e-5, pressure after one Jacobi update 3.4e-6 and after
1 / 3 / 10 sweeps 4.8e-5 / 4.4e-5 / 6.1e-5; FP64 error sums 3.2e-9 relative.
"""
import numpy as np
import pytest

from oracle import OracleBackend
from parity_util import assert_neighbor_structures_equal, elementwise_errors, report
from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import SimBackendB200

pytestmark = pytest.mark.gpu

DEVELOP_STEPS = 200
FIELDS = (abi.FIELD_DENSITY, abi.FIELD_VEL_PRED, abi.FIELD_SOURCE, abi.FIELD_DIAG, abi.FIELD_PRESSURE,
          abi.FIELD_ACC_PRESS)
G = 9.81

# (stage, output fields)
STAGES = ((abi.STAGE_DENSITY, (abi.FIELD_DENSITY,)),
          (abi.STAGE_NON_PRESSURE, (abi.FIELD_VEL_PRED,)),
          (abi.STAGE_SOURCE_DIAG_INIT, (abi.FIELD_SOURCE, abi.FIELD_DIAG, abi.FIELD_PRESSURE)),
          (abi.STAGE_PRESSURE_ACC, (abi.FIELD_ACC_PRESS,)),
          (abi.STAGE_JACOBI_UPDATE, (abi.FIELD_PRESSURE,)))


def floors(diag_scale, acc_scale):
    return {abi.FIELD_DENSITY: 1e-3, abi.FIELD_VEL_PRED: 1e-5 * G * 5e-4, abi.FIELD_SOURCE: 1e-3,
            abi.FIELD_DIAG: 1e-6 * diag_scale, abi.FIELD_PRESSURE: 1e-2, abi.FIELD_ACC_PRESS: 1e-6 * acc_scale}


# element-wise relative bound against the FP32 oracle, per field (floors above)
RTOL_FP32 = {abi.FIELD_DENSITY: 2e-6, abi.FIELD_VEL_PRED: 2e-6, abi.FIELD_SOURCE: 1e-4, abi.FIELD_DIAG: 2e-5,
             abi.FIELD_PRESSURE: 1e-4, abi.FIELD_ACC_PRESS: 1e-4}
RTOL_FP64 = 1e-4  # per-step field error against FP64 <= 1e-4 relative
JACOBI_SWEEPS = (1, 3, 10)


@pytest.fixture(scope="module")
def developed():
    st, dmin, dmax, p = S.dam_1m()
    g = SimBackendB200(p)
    g.set_sim_domain_bounds(dmin, dmax)
    g.pull(st, p)
    g.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    g.step(p, DEVELOP_STEPS)
    dev = g.push()
    g.close()
    return dev, dmin, dmax, p


def _load(be, st, p, dmin, dmax):
    be.set_sim_domain_bounds(dmin, dmax)
    be.pull(st, p)
    be.neighbor_search(p)
    return be


def stage_reports(developed):
    """Runs every stage from identical inputs on the GPU, the FP32 and the FP64 oracle; returns
    {name: (summary vs FP32, summary vs FP64)} and the bit-exact structure check's backends."""
    st, dmin, dmax, p = developed
    g = _load(SimBackendB200(p), st, p, dmin, dmax)
    o = _load(OracleBackend(p), st, p, dmin, dmax)
    d = _load(OracleBackend(p, fp64=True), st, p, dmin, dmax)
    # FP64 frame arithmetic may order a particle on a cell boundary differently: align by ID
    ids_o, ids_d = o.push().idF, d.push().idF
    assert np.array_equal(g.push().idF, ids_o)
    to_d = np.argsort(ids_o)[np.searchsorted(ids_o[np.argsort(ids_o)], ids_d)]  # d order -> o index
    from_d = np.argsort(to_d)
    diag_scale = acc_scale = None
    out = {}
    for stage, fields in STAGES:
        for f in FIELDS:
            v = o.read_field(f)
            g.write_field(f, v)
            d.write_field(f, v[to_d])
        eg, eo, ed = g.run_stage(stage, p), o.run_stage(stage, p), d.run_stage(stage, p)
        for f in fields:
            a, b, c = g.read_field(f), o.read_field(f), d.read_field(f)[from_d]
            if diag_scale is None and f == abi.FIELD_DIAG:
                diag_scale = float(np.abs(c).max())
            if acc_scale is None and f == abi.FIELD_ACC_PRESS:
                acc_scale = float(np.abs(c).max())
            fl = floors(diag_scale or 1.0, acc_scale or 1.0)[f]
            out[f"stage{stage}_field{f}"] = (elementwise_errors(a, b, RTOL_FP32[f], fl)[1],
                                             elementwise_errors(a, c, RTOL_FP64, fl)[1])
        if stage == abi.STAGE_JACOBI_UPDATE:
            out["jacobi_error_sums"] = (elementwise_errors(eg, eo, 1e-9, 0.0)[1],
                                        elementwise_errors(eg, ed, 1e-6, 0.0)[1])
    # pressure after k relaxed-Jacobi sweeps from one identical initial state (source/diagonal
    # stage of each backend on identical inputs, then k x (pressure acceleration, Jacobi update))
    for f in FIELDS:
        v = o.read_field(f)
        g.write_field(f, v)
        d.write_field(f, v[to_d])
    for be in (g, o, d):
        be.run_stage(abi.STAGE_SOURCE_DIAG_INIT, p)
    done = 0
    for k in JACOBI_SWEEPS:
        for _ in range(k - done):
            for be in (g, o, d):
                be.run_stage(abi.STAGE_PRESSURE_ACC, p)
                be.run_stage(abi.STAGE_JACOBI_UPDATE, p)
        done = k
        a, b, c = (g.read_field(abi.FIELD_PRESSURE), o.read_field(abi.FIELD_PRESSURE),
                   d.read_field(abi.FIELD_PRESSURE)[from_d])
        # k sweeps compound the FP32 rounding of each: the bounds grow with k
        out[f"pressure_after_{k}_sweeps"] = (elementwise_errors(a, b, RTOL_FP32[abi.FIELD_PRESSURE] * k, 1e-2 * k)[1],
                                             elementwise_errors(a, c, RTOL_FP64 * k, 1e-2 * k)[1])
    return out, (g, o)


@pytest.fixture(scope="module")
def reports(developed):
    r = stage_reports(developed)
    report("dam_1m_stages", r[0])
    return r


def test_dam_1m_developed_neighbor_structures_bit_exact(developed, reports):
    st = developed[0]
    g, o = reports[1]
    assert_neighbor_structures_equal(g, o, st.N_F, st.N_B, st.N_R)


@pytest.mark.parametrize("which", ["fp32", "fp64"])
def test_dam_1m_stages_elementwise(reports, which):
    k = 0 if which == "fp32" else 1
    bad = {name: s[k] for name, s in reports[0].items() if s[k]["bad"]}
    assert not bad, f"element-wise bound exceeded against the {which} oracle: {bad}"
