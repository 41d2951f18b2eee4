"""Known-answer cases restated from the reference's own unit tests.

Every case cites the reference test it comes from (paths relative to the reference repo).
Scenes are built as UniversalSimState objects so the same case drives the CPU oracle and
the B200 backend through identical method calls.
"""
from __future__ import annotations

import math

import numpy as np

from turbospharticles_b200 import abi
from turbospharticles_b200.params import SimParams
from turbospharticles_b200.state import UniversalSimState

f32 = np.float32


# ------------------------------------------------------------------------- neighbor search
def ns_params(ratio=1.0):
    """tests/unit/neighbor_search.cpp:180-195: h = 0.5, r = 1, massF = massB = 125."""
    return SimParams(particleSizeF=0.5, particleSizeB=0.5, kernelRadius=1.0, kernelRadiusSqu=1.0,
                     massF=125.0, massB=125.0, gridCellSizeRatio=ratio)


def make_particles(fluid, boundary=(), rigid=(), body_ids=None):
    """MakeParticles + MakeState (neighbor_search.cpp:43-115): descending noncontiguous IDs,
    identity orientation, zero centre of mass (relative == world rigid positions)."""
    pops = [list(fluid), list(boundary), list(rigid)]
    ids = [np.array([5_000_000_000 * (p + 1) + 17 * (len(pops[p]) - i) for i in range(len(pops[p]))],
                    np.uint64) for p in range(3)]
    bodies = (np.array(body_ids, np.uint32) if body_ids is not None
              else np.arange(len(pops[2]), dtype=np.uint32))
    n_bodies = int(bodies.max()) + 1 if len(pops[2]) else 0
    st = UniversalSimState(len(pops[0]), len(pops[1]), len(pops[2]), n_bodies)
    st.idF[:] = ids[0]; st.idB[:] = ids[1]; st.idR[:] = ids[2]
    for arr, pts in ((("xPosF", "yPosF", "zPosF"), pops[0]), (("xPosB", "yPosB", "zPosB"), pops[1]),
                     (("xPosRelR", "yPosRelR", "zPosRelR"), pops[2])):
        P = np.array(pts, f32).reshape(-1, 3)
        for a in range(3):
            getattr(st, arr[a])[:] = P[:, a]
    st.volB[:] = 1.0; st.psiB[:] = 1000.0
    st.volR[:] = 1.0; st.psiR[:] = 1000.0
    st.bodyIdR[:] = bodies[:len(pops[2])]
    st.massRB[:] = 1.0; st.massInvRB[:] = 1.0
    st.iBodyInv00[:] = 1.0; st.iBodyInv11[:] = 1.0; st.iBodyInv22[:] = 1.0
    for b in range(n_bodies):
        st.rigidParticleCountRB[b] = int((bodies == b).sum())
    return st


def _nf(x, toward):
    return float(np.nextafter(f32(x), f32(toward)))


INSIDE = _nf(1.0, 0.0)
OUTSIDE = _nf(1.0, 2.0)

NS_SCENES = {
    # neighbor_search.cpp:214-229
    "mixed": dict(fluid=[(3, 0, 0), (-0.25, 0, 0), (0.5, 0.25, 0), (-3, 1, 0), (0.25, -0.5, 0.25)],
                  boundary=[(-3, 0.5, 0), (0, 0, 0), (3.5, 0.25, 0), (6, 6, 6)],
                  rigid=[(0.25, 0.25, 0.25), (-0.5, 0.25, 0), (3.25, 0, 0), (-3, 1.5, 0)],
                  body_ids=[0, 0, 1, 2]),
    # :232-243
    "cutoff": dict(fluid=[(OUTSIDE, 0, 0), (0, 0, 0), (INSIDE, 0, 0), (1, 0, 0)],
                   boundary=[(-OUTSIDE, 0, 0), (-1, 0, 0), (-INSIDE, 0, 0), (0, 0, 0)],
                   rigid=[(1, 0, 0), (OUTSIDE, 0, 0), (INSIDE, 0, 0), (-1, 0, 0)]),
    # :245-250
    "off_axis": dict(fluid=[(0, 0, 0), (0.1, 0.3, 0.94868332)], boundary=[(0, 0, 0), (0.1, 0.3, 0.94868332)],
                     rigid=[(0, 0, 0), (0.1, 0.3, 0.94868332)]),
    # :252-263
    "cell_boundaries": dict(
        fluid=[(-0.125, -0.125, -0.125), (0.125, -0.125, -0.125), (0.125, 0.125, -0.125), (0.125, 0.125, 0.125),
               (-1.125, -0.125, 0.125), (-0.875, 0.125, -0.125), (2.125, 2.125, 2.125)],
        boundary=[(0.875, -0.125, 0.125), (1.125, 0.125, -0.125), (-0.125, 0.125, 0.125)],
        rigid=[(-0.125, 0.125, -0.125), (0.125, -0.125, 0.125)]),
    # :265-278 (also searched with cell size ratios 0.5, 0.25, 1.0)
    "small_cells": dict(fluid=[(0.125, 0.125, 0.125), (0.875, 0.125, 0.125), (-0.625, 0.125, 0.125),
                               (2.125, 0.125, 0.125)],
                        boundary=[(0.125, 0.875, 0.125), (0.125, -0.625, 0.125)],
                        rigid=[(0.125, 0.125, 0.875), (0.125, 0.125, -0.625)]),
    # :298-308
    "coincident": dict(fluid=[(0, 0, 0), (0, 0, 0)], boundary=[(0, 0, 0)], rigid=[(0, 0, 0)] * 4,
                       body_ids=[0, 0, 1, 1]),
    # :280-296
    "empty": dict(fluid=[]),
    "fluid_only": dict(fluid=[(2, 0, 0), (-2, 0, 0)]),
    "boundary_only": dict(fluid=[], boundary=[(0, 0, 0), (0.5, 0, 0)]),
    "rigid_only": dict(fluid=[], rigid=[(0, 0, 0), (0.5, 0, 0)]),
}


def simd_width_scene(n_f):
    """neighbor_search.cpp:310-328 (counts around the CPU SIMD width, here also around 32)."""
    fluid = [(0.25 * (i % 5) - 0.5, 0.25 * (i // 5), 0.125 if i % 2 == 0 else -0.125) for i in range(n_f)]
    return dict(fluid=fluid, boundary=[(-0.25, 0.25, 0), (0.5, 0.5, 0.25)],
                rigid=[(0.25, 0.25, 0.25), (-0.5, 0.5, -0.25)])


def dense_lattice_scene(n_f):
    """neighbor_search.cpp:330-345: every pair within the cutoff."""
    fluid = [(0.08 * (i % 7), 0.08 * ((i // 7) % 7), 0.08 * (i // 49)) for i in range(n_f)]
    return dict(fluid=fluid, boundary=[(0.25, 0.25, -0.25)], rigid=[(0.25, -0.25, 0.25)])


def reference_neighbors(scene, radius_squ=1.0):
    """Independent FP64 all-pairs reference (neighbor_search.cpp:118-137): sorted neighbor-ID
    lists per category FF, FB, FR, RF, RB, RR, keyed by source ID."""
    st = make_particles(**scene)
    pos = [np.stack([st.xPosF, st.yPosF, st.zPosF], 1).astype(np.float64),
           np.stack([st.xPosB, st.yPosB, st.zPosB], 1).astype(np.float64),
           np.stack([st.xPosRelR, st.yPosRelR, st.zPosRelR], 1).astype(np.float64)]
    ids = [st.idF, st.idB, st.idR]
    out = {}
    for cat, (s, t) in enumerate(((0, 0), (0, 1), (0, 2), (2, 0), (2, 1), (2, 2))):
        res = {}
        for a in range(len(ids[s])):
            nb = []
            for b in range(len(ids[t])):
                if s == 2 and t == 2 and st.bodyIdR[a] == st.bodyIdR[b]:
                    continue
                d = pos[s][a] - pos[t][b]
                if d[0] * d[0] + d[1] * d[1] + d[2] * d[2] <= radius_squ:
                    nb.append(int(ids[t][b]))
            res[int(ids[s][a])] = sorted(nb)
        out[cat] = res
    return out


def backend_neighbors(be, st_pushed):
    """Neighbor-ID lists by category from a backend after a search (IDs via the pushed state)."""
    ids = [st_pushed.idF, st_pushed.idB, st_pushed.idR]
    out = {}
    for cat, (s, t) in enumerate(((0, 0), (0, 1), (0, 2), (2, 0), (2, 1), (2, 2))):
        off, idx = be.rows(cat)
        res = {}
        for a in range(len(ids[s])):
            row = idx[int(off[a]):int(off[a + 1])]
            res[int(ids[s][a])] = sorted(int(ids[t][j]) for j in row)
        out[cat] = res
    return out


# ------------------------------------------------------------------------- SPH stage KATs
def pressure_params():
    """tests/unit/sph_pressure.cpp:47-61 (+ alpha = 1/4 of the test fixture, :386)."""
    return SimParams(timeStep=0.5, particleSizeF=1.0, particleSizeB=1.0, kernelRadius=2.0,
                     kernelRadiusSqu=4.0, restDensity=1.0, massF=1.0, massB=1.0, pressGamma=0.375,
                     jacobiOmega=0.25, gravity=(0.0, 0.0, 0.0), cubicSplineAlphaOverride=0.25)


def fluid_pair_state(density=9.0 / 8.0):
    """MakeFluidPair (sph_pressure.cpp:69-76): stationary pair at x = -+0.25."""
    st = UniversalSimState(2, 0, 0, 0, 1.0)
    st.xPosF[:] = [-0.25, 0.25]
    st.densityF[:] = density
    return st


PRESSURE_KATS = dict(source=-1.0 / 8.0, diag=-225.0 / 512.0, pressure=16.0 / 225.0, acc=2.0 / 15.0,
                     jacobi=24.0 / 225.0, err=1.0 / 8.0)


def kat_tol(expected):
    """ExpectPressureNear (sph_pressure.cpp:183)."""
    return 1e-7 + 5e-6 * abs(expected)


def kernel_reference(offset, h):
    """ReferenceKernel (tests/unit/sph_kernels.cpp:73-98), FP64 closed form."""
    d = np.asarray(offset, np.float64)
    dist = math.sqrt(float(d @ d))
    q = dist / h
    if q >= 2.0:
        return 0.0, np.zeros(3)
    norm = 1.0 / (math.pi * h ** 3)
    shape = 1.0 - 1.5 * q * q + 0.75 * q ** 3 if q < 1.0 else 0.25 * (2.0 - q) ** 3
    deriv = -3.0 * q + 2.25 * q * q if q < 1.0 else -0.75 * (2.0 - q) ** 2
    g = d * (norm * deriv / (h * dist)) if dist > 0 else np.zeros(3)
    return norm * shape, g


def alpha_of(h):
    """BuildSolverConstants alpha (solver_constants.h:287-303)."""
    inv = 1.0 / float(f32(h))
    return float(f32(inv * inv * inv / (4.0 * math.pi)))


def pressure_pair_kats(be):
    """Runs the sph_pressure.cpp KATs (:391-463) through a backend's stage API; returns the
    measured values keyed like PRESSURE_KATS. The search-built lists contain each particle's
    self pair in addition to the tests' hand lists; a self pair contributes exactly zero."""
    p = pressure_params()
    be.pull(fluid_pair_state(), p)
    be.neighbor_search(p)
    be.write_field(abi.FIELD_DENSITY, np.full(2, 9.0 / 8.0))
    be.run_stage(abi.STAGE_SOURCE_DIAG_INIT, p)
    out = dict(source=be.read_field(abi.FIELD_SOURCE), diag=be.read_field(abi.FIELD_DIAG),
               pressure=be.read_field(abi.FIELD_PRESSURE))
    # warm start (:405-420)
    pw = p.copy(jacobiWarmStart=0.5)
    ids = be.push().idF
    prev = np.where(ids == ids.min(), 0.25, 0.125)  # first listed particle gets 0.25
    be.write_field(abi.FIELD_PRESSURE, prev)
    be.run_stage(abi.STAGE_SOURCE_DIAG_INIT, pw)
    out["warm"] = (be.read_field(abi.FIELD_PRESSURE), prev)
    # pair acceleration (:422-436)
    be.write_field(abi.FIELD_PRESSURE, np.full(2, 16.0 / 225.0))
    be.run_stage(abi.STAGE_PRESSURE_ACC, p)
    acc = be.read_field(abi.FIELD_ACC_PRESS)
    x = be.read_field(abi.FIELD_POS)
    out["acc"] = (acc, x)
    # Jacobi update with known accelerations (:438-452)
    be.write_field(abi.FIELD_SOURCE, np.full(2, -1.0 / 8.0))
    be.write_field(abi.FIELD_DIAG, np.full(2, -225.0 / 512.0))
    a = np.zeros((2, 3))
    a[:, 0] = np.where(x[:, 0] < 0, -2.0 / 15.0, 2.0 / 15.0)
    be.write_field(abi.FIELD_ACC_PRESS, a)
    be.write_field(abi.FIELD_PRESSURE, np.full(2, 16.0 / 225.0))
    err = be.run_stage(abi.STAGE_JACOBI_UPDATE, p)
    out["jacobi"] = be.read_field(abi.FIELD_PRESSURE)
    out["err"] = err
    return out


def check_pressure_pair(out):
    K = PRESSURE_KATS
    for i in range(2):
        assert abs(out["source"][i] - K["source"]) <= kat_tol(K["source"])
        assert abs(out["diag"][i] - K["diag"]) <= kat_tol(K["diag"])
        assert abs(out["pressure"][i] - K["pressure"]) <= kat_tol(K["pressure"])
    warm, prev = out["warm"]
    for i in range(2):
        assert abs(warm[i] - 0.5 * prev[i]) <= kat_tol(0.5 * prev[i])
    acc, x = out["acc"]
    for i in range(2):
        exp = -K["acc"] if x[i, 0] < 0 else K["acc"]
        assert abs(acc[i, 0] - exp) <= kat_tol(exp)
        assert acc[i, 1] == 0.0 and acc[i, 2] == 0.0
    for v in out["jacobi"]:
        assert abs(v - K["jacobi"]) <= kat_tol(K["jacobi"])
    for e in out["err"]:
        assert abs(e - K["err"]) <= kat_tol(K["err"])


def integration_kats():
    """tests/unit/sph_integration.cpp:101-150: (pos, velPred, accPress, dt) -> (pos, vel), exact."""
    return [
        (((1, -4, 10), (3, -2, 0.5), (4, 8, -6)), 0.25, ((2, -4, 9.75), (4, 0, -1))),
        (((1, -2, 3), (2, -4, 6), (0, 0, 0)), 0.5, ((2, -4, 6), (2, -4, 6))),
        (((-7, 8, -9), (0, 0, 0), (0, 0, 0)), 0.5, ((-7, 8, -9), (0, 0, 0))),
        (((1, -4, 10), (3, -2, 0.5), (4, 8, -6)), 0.0, ((1, -4, 10), (3, -2, 0.5))),
    ]


def density_kat_state():
    """sph_density.cpp:233-243: fluid at (0,0,0), (1,0,0), (0,1.5,0), h = 1, massF = 2; the
    first particle's list {2, 0, 1} is its full search neighborhood -> 10.25 / (4 pi)."""
    p = SimParams(particleSizeF=1.0, particleSizeB=1.0, kernelRadius=2.0, kernelRadiusSqu=4.0, massF=2.0,
                  restDensity=1000.0)
    st = UniversalSimState(3, 0, 0, 0)
    st.xPosF[:] = [0.0, 1.0, 0.0]
    st.yPosF[:] = [0.0, 0.0, 1.5]
    return st, p, 10.25 / (4.0 * math.pi)


def viscosity_kat_state(massF, densityJ):
    """sph_non_pressure.cpp:309-331: pair at one smoothing length; the first particle's
    predicted x-velocity drops by 3 m / (16 pi rho_j 1.01)."""
    p = SimParams(timeStep=0.125, particleSizeF=1.0, particleSizeB=1.0, kernelRadius=2.0, kernelRadiusSqu=4.0,
                  massF=massF, viscosityF=0.1, viscosityB=0.2, gravity=(0.0, 0.0, 0.0))
    st = UniversalSimState(2, 0, 0, 0)
    st.xPosF[:] = [0.0, 1.0]
    st.xVelF[:] = [1.0, -1.0]
    st.yVelF[:] = [2.0, 2.0]
    st.zVelF[:] = [3.0, 3.0]
    st.densityF[:] = [9.0, densityJ]
    return st, p, 1.0 - 3.0 * massF / (16.0 * math.pi * densityJ * 1.01)
