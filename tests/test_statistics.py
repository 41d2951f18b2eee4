"""Statistics record (FillStatisticsRecord, source/simulation/GPU/backend/gpu_backend.cpp:
1067-1203; Stats::StatMetric, source/eval/stats/metrics.h:23-86) of the oracle, checked on the
CPU against the same quantities recomputed from its neighbor rows and pushed state."""
import numpy as np

from oracle import OracleBackend
from turbospharticles_b200 import abi, scene as S


def test_oracle_statistics_record():
    st, dmin, dmax, p = S.floating_cubes()
    o = OracleBackend(p)
    o.set_sim_domain_bounds(dmin, dmax)
    o.pull(st, p)
    o.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    o.step(p)
    rec = o.statistics(p)
    assert list(rec) == list(abi.STAT_NAMES) and len(rec) == 35
    out = o.push()
    assert rec["NumF"] == st.N_F and rec["NumB"] == st.N_B and rec["NumR"] == st.N_R
    for k, rel in enumerate(("FF", "FB", "FR", "RF", "RB", "RR")):
        off, _ = o.rows(k)
        cnt = np.diff(off.astype(np.int64))
        srt = np.sort(cnt)
        assert rec[f"NumNbr{rel}_Avg"] == cnt.sum() / cnt.size
        assert rec[f"NumNbr{rel}_Min"] == srt[0] and rec[f"NumNbr{rel}_Max"] == srt[-1]
        assert rec[f"NumNbr{rel}_P99"] == srt[(99 * (cnt.size - 1)) // 100]
    rel = (out.densityF / np.float32(p.restDensity)).astype(np.float32) - np.float32(1.0)
    assert abs(rec["DensRelError_Raw_Avg"] - float(np.mean(rel.astype(np.float64)))) <= 1e-12
    assert abs(rec["DensRelError_Pos_Avg"] - float(np.mean(np.maximum(rel, 0).astype(np.float64)))) <= 1e-12
    v = np.sqrt((out.xVelF * out.xVelF + out.yVelF * out.yVelF + out.zVelF * out.zVelF).astype(np.float32))
    assert np.isclose(rec["VelMag_Max"], float(v.max()), rtol=1e-6)
    assert np.isclose(rec["CFL_Number"], float(np.float32(v.max()) * np.float32(p.timeStep) / np.float32(p.particleSizeF)),
                      rtol=1e-6)
    assert rec["NumSolverIters"] == o.stats().solverIters
