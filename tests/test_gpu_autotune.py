"""The autotuner (tune.cu): every tuned kernel gets a recorded choice on the first step, the
choice is one of its candidates and no slower than the untuned configuration it was timed
against, and tuned runs are bit-identical to untuned ones (candidates differ in registers and
load grouping, never in the order of a sum)."""
import numpy as np
import pytest

from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import SimBackendB200

pytestmark = pytest.mark.gpu

TUNED = ("KDensity", "KNonPressure", "KSourceDiagInit", "KPressureAcc", "KJacobi", "KQueryFluidCount",
         "KQueryFluidFill")


def run(steps, autotune):
    abi.reset_tuning()
    abi.set_autotune(autotune)
    try:
        st, dmin, dmax, p = S.dam_32k()
        g = SimBackendB200(p)
        g.set_sim_domain_bounds(dmin, dmax)
        g.pull(st, p)
        g.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
        g.step(p, steps)
        return g.push(), abi.tuning(0)
    finally:
        abi.set_autotune(True)


def test_autotune_choices_recorded_and_results_bit_identical():
    tuned, report = run(8, True)
    plain, report_off = run(8, False)
    assert report_off == {}
    names = {k.split("/")[0] for k in report}
    assert set(TUNED) <= names, report
    for k, v in report.items():
        assert 0 < v["min_blocks"] <= 32 and v["candidates"] >= 2, (k, v)
        assert v["ms"] <= v["untuned_ms"] + 1e-6, (k, v)
    for name in ("xPosF", "yPosF", "zPosF", "xVelF", "pressureF", "densityF", "idF"):
        assert np.array_equal(getattr(tuned, name), getattr(plain, name)), name
