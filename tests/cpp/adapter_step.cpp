// Drives the B200 backend through the C++ adapter (include/tsp_b200_backend.hpp) the way the
// reference's SimulationMgr drives I_SimBackend: pull, neighbor search, steps, push.
// A 16^3 fluid lattice in free fall (no walls) must fall by g t^2 / 2 to FP32 accuracy; the
// statistics record and the export snapshot come through the same adapter.
#include <cmath>
#include <cstdio>
#include <vector>

#include "tsp_b200_backend.hpp"

int main() {
    const uint32_t n = 16, N = n * n * n;
    const float h = 0.02f, dt = 1e-3f;
    tsp_params p{};
    p.timeStep = dt; p.particleSizeF = h; p.particleSizeB = h;
    p.kernelRadius = 2.0f * h; p.kernelRadiusSqu = p.kernelRadius * p.kernelRadius;
    p.restDensity = 1000.0f; p.massF = 1000.0f * h * h * h; p.massB = p.massF;
    p.viscosityF = 0.0f; p.viscosityB = 0.0f; p.gravity[1] = -9.81f;
    p.pressGamma = 0.5f; p.jacobiOmega = 0.5f; p.densityDevTarget = 0.001f;
    p.minSolverIters = 2; p.maxSolverIters = 100; p.solverTerminationCond = TSP_TERM_REL_ERR_POS;
    p.gridCellSizeRatio = 1.0f; p.boundaryLayers = 2;
    std::vector<uint64_t> id(N);
    std::vector<float> x(N), y(N), z(N), dens(N, 1000.0f);
    for (uint32_t k = 0; k < N; k++) {
        id[k] = k;
        x[k] = h * (k % n); y[k] = 1.0f + h * ((k / n) % n); z[k] = h * (k / (n * n));
    }
    tsp_state_view v{};
    v.N_F = N; v.idF = id.data(); v.xPosF = x.data(); v.yPosF = y.data(); v.zPosF = z.data(); v.densityF = dens.data();
    try {
        tsp::SimBackendB200 be(p, 0);
        be.PullFromUniversalSimState(v, p);
        be.ExecuteNeighborSearch(p);
        const int steps = 5;
        for (int s = 0; s < steps; s++) be.ExecuteFullSimStep(p);
        std::vector<uint64_t> id2(N);
        std::vector<float> x2(N), y2(N), z2(N);
        tsp_state_view o{};
        o.idF = id2.data(); o.xPosF = x2.data(); o.yPosF = y2.data(); o.zPosF = z2.data();
        be.PushToUniversalSimState(o);
        double yMean0 = 0, yMean1 = 0;
        for (uint32_t k = 0; k < N; k++) { yMean0 += y[k]; yMean1 += y2[k]; }
        yMean0 /= N; yMean1 /= N;
        // semi-implicit Euler: y_n = y_0 - g dt^2 n (n + 1) / 2 for the centre of mass
        const double expected = -9.81 * dt * dt * steps * (steps + 1) / 2.0;
        const double got = yMean1 - yMean0;
        std::printf("%s N=%u steps=%d dy=%.9g expected=%.9g iters=%u\n", be.Name(), be.GetNumFluidParticles(), steps,
                    got, expected, be.Stats().solverIters);
        if (std::fabs(got - expected) > 2e-2 * std::fabs(expected)) return 2;  // FP32 position rounding
        if (o.N_F != N || be.Stats().step != (uint64_t)steps) return 3;
        double rec[TSP_STAT_COUNT];
        be.FillStatisticsRecord(p, rec);
        const double vExpected = 9.81 * dt * steps;  // every particle falls at the same speed
        std::printf("NumF=%g VelMag_Avg=%.9g expected=%.9g\n", rec[TSP_STAT_NUM_F], rec[TSP_STAT_VEL_MAG_AVG], vExpected);
        if (rec[TSP_STAT_NUM_F] != N || std::fabs(rec[TSP_STAT_VEL_MAG_AVG] - vExpected) > 2e-2 * vExpected) return 4;
        std::vector<float> ex(N), ey(N), ez(N), ev(N);
        tsp_export_snapshot snap{};
        snap.xPosF = ex.data(); snap.yPosF = ey.data(); snap.zPosF = ez.data(); snap.velMagF = ev.data();
        be.PackExportSnapshot(snap, p, false);
        std::printf("exported %u of %u fluid particles\n", snap.N_F, N);
        if (snap.N_F == 0 || snap.N_F > N || snap.N_B != 0 || snap.simStep != (uint64_t)steps) return 5;
    } catch (const std::exception& e) {
        std::printf("error: %s\n", e.what());
        return 1;
    }
    return 0;
}
