"""SimParams: the subset of the reference's `Sim::SimParams` that the IISPH step reads.

Field names and defaults follow source/simulation/core/parameters_sim.h:25-175; derived
values follow the setters in source/simulation/core/parameters_sim.cpp:1478-1483,1497-1501
(massF = restDensity * h^3, kernelRadius = kernelSuppRatio * h, kernelRadiusSqu = r^2).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .abi import TspParams, TERM_FIXED_ITERS

CUBIC_SPLINE_SUPP_RATIO = 2.0  # parameters_sim.h:22


@dataclasses.dataclass
class SimParams:
    timeStep: float = 0.0001
    particleSizeF: float = 0.01
    particleSizeB: float = 0.01
    kernelSuppRatio: float = CUBIC_SPLINE_SUPP_RATIO
    kernelRadius: float = 0.02
    kernelRadiusSqu: float = 0.0004
    restDensity: float = 1000.0
    massF: float = 0.001
    massB: float = 0.001
    viscosityF: float = 0.00001
    viscosityB: float = 0.00001
    gravity: tuple = (0.0, -9.81, 0.0)
    pressGamma: float = 0.5
    jacobiOmega: float = 0.6
    jacobiWarmStart: float = 0.0
    densityDevTarget: float = 0.01
    fixedIters: int = 10
    minSolverIters: int = 5
    maxSolverIters: int = 50
    solverTerminationCond: int = TERM_FIXED_ITERS
    gridCellSizeRatio: float = 1.0
    boundaryLayers: int = 2
    cubicSplineAlphaOverride: float = 0.0
    rigidContactDensityDevTarget: float = 0.001   # parameters_sim.h:100
    rigidContactMaxSolverIters: int = 100         # parameters_sim.h:101
    surfaceNbrCountThreshold: int = 27            # parameters_sim.h:170 (export surface classification)
    # mesh surface sampling (parameters_sim.h:122-139); the distances follow the ratios x
    # particleSizeB (UpdateSurfaceSamplingDistances_, parameters_sim.cpp:2032-2046)
    surfaceSamplingMinDistanceRatioB: float = 0.8
    surfaceSamplingMaxDistanceRatioB: float = 1.0
    surfaceSamplingCoverageProbeSpacingRatioB: float = 0.2
    surfaceSamplingMinDistanceRatioR: float = 0.8
    surfaceSamplingMaxDistanceRatioR: float = 1.0
    surfaceSamplingCoverageProbeSpacingRatioR: float = 0.2
    surfaceSamplingMinDistanceB: float = 0.008
    surfaceSamplingMaxDistanceB: float = 0.01
    surfaceSamplingCoverageProbeSpacingB: float = 0.002
    surfaceSamplingMinDistanceR: float = 0.008
    surfaceSamplingMaxDistanceR: float = 0.01
    surfaceSamplingCoverageProbeSpacingR: float = 0.002
    surfaceSamplingCandidateMultiplier: int = 8
    surfaceSamplingSeed: int = 42
    # scene-building parameters (builder.cpp; not read by the step)
    jitterFracF: float = 0.0
    jitterSeedF: int = 42
    jitterFracB: float = 0.0
    jitterSeedB: int = 42

    def set_particle_size(self, h: float) -> "SimParams":
        """Set_ParticleSize for fluid and boundary (parameters_sim.cpp:1476-1501), FP32."""
        f32 = np.float32
        h32 = f32(h)
        self.particleSizeF = float(h32)
        self.particleSizeB = float(h32)
        self.massF = float(f32(f32(f32(f32(self.restDensity) * h32) * h32) * h32))
        self.massB = self.massF
        self.kernelRadius = float(f32(f32(self.kernelSuppRatio) * h32))
        self.kernelRadiusSqu = float(f32(f32(self.kernelRadius) * f32(self.kernelRadius)))
        for kind in ("B", "R"):
            for q in ("MinDistance", "MaxDistance", "CoverageProbeSpacing"):
                ratio = f32(getattr(self, f"surfaceSampling{q}Ratio{kind}"))
                setattr(self, f"surfaceSampling{q}{kind}", float(f32(ratio * f32(self.particleSizeB))))
        return self

    def set_rest_density(self, rho: float) -> "SimParams":
        self.restDensity = float(np.float32(rho))
        return self.set_particle_size(self.particleSizeF)

    def to_c(self) -> TspParams:
        p = TspParams()
        for f in ("timeStep", "particleSizeF", "particleSizeB", "kernelRadius", "kernelRadiusSqu",
                  "restDensity", "massF", "massB", "viscosityF", "viscosityB", "pressGamma",
                  "jacobiOmega", "jacobiWarmStart", "densityDevTarget", "fixedIters",
                  "minSolverIters", "maxSolverIters", "solverTerminationCond",
                  "gridCellSizeRatio", "boundaryLayers", "cubicSplineAlphaOverride",
                  "rigidContactDensityDevTarget", "rigidContactMaxSolverIters", "surfaceNbrCountThreshold"):
            setattr(p, f, getattr(self, f))
        for a in range(3):
            p.gravity[a] = self.gravity[a]
        return p

    def copy(self, **kw) -> "SimParams":
        return dataclasses.replace(self, **kw)


def dam_params(dx: float, dt: float, omega: float = 0.5, min_iters: int = 2,
               max_iters: int = 100, target: float = 0.001, term: int = 2) -> SimParams:
    """Physics of the dam-break workloads: cubic spline support 2*dx, rho0 = 1000,
    g = -9.81 (y), relaxed Jacobi with omega, average density-error termination
    (RelDensityError_Pos by default), viscosities of configs/params_def.json."""
    p = SimParams(timeStep=dt, viscosityF=0.00004, viscosityB=0.00008, pressGamma=0.5,
                  jacobiOmega=omega, jacobiWarmStart=0.0, densityDevTarget=target,
                  minSolverIters=min_iters, maxSolverIters=max_iters,
                  solverTerminationCond=term, boundaryLayers=2)
    return p.set_particle_size(dx)
