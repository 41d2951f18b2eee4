"""Mesh surface sampling on the GPU (tsp_b200_sample_surface) and mesh-built scenes.

- The GPU sampler returns exactly the oracle's samples (same order, same FP32 bits) and the
  same statistics on curved, axis-aligned, thin and larger meshes, and rejects what the oracle
  rejects.
- A mesh rigid body (sampled icosphere) floating on the fluid and a mesh boundary obstacle
  (sampled box) step on the GPU like the oracle: centre of mass within 1e-5 m, body velocity
  within 1e-4 m/s after 10 steps; fluid positions within 1e-5 m.
"""
import numpy as np
import pytest

import oracle
from oracle import OracleBackend
from turbospharticles_b200 import abi, mesh as M, scene as S
from turbospharticles_b200.backend import SimBackendB200
from turbospharticles_b200.params import SimParams
from turbospharticles_b200.state import BOUNDARY_F32, FLUID_F32, UniversalSimState

pytestmark = pytest.mark.gpu


def tetra(extent):
    m = M.TriangleSurfaceMesh(np.array([(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)], np.float32),
                              np.array([(0, 2, 1), (0, 1, 3), (0, 3, 2), (1, 2, 3)], np.uint32))
    M.scale_to_target_extent(m, extent)
    return m


CASES = [("sphere", lambda: M.icosphere(0.1, 2), 0.02), ("box", lambda: M.box_mesh((0.1, 0.06, 0.04)), 0.02),
         ("thin box", lambda: M.box_mesh((0.2, 0.01, 0.15)), 0.01), ("tetra", lambda: tetra(0.15), 0.02),
         ("large sphere", lambda: M.icosphere(0.5, 3), 0.01)]


@pytest.mark.parametrize("name,make,h", CASES, ids=[c[0] for c in CASES])
def test_gpu_sampler_matches_oracle(name, make, h):
    mesh = make()
    sp = M.sampling_params(SimParams().set_particle_size(h), "R")
    g, gs = M.sample_surface(mesh, sp)
    o, os_ = oracle.sample_surface(mesh, sp)
    assert len(g) == len(o) > 0
    np.testing.assert_array_equal(g.view(np.uint32), o.view(np.uint32))
    for f in ("N_candidates", "N_initialSamples", "N_coverageRepairs", "N_coverageProbes", "surfaceArea"):
        assert getattr(gs, f) == getattr(os_, f), f


def test_gpu_sampler_seed_changes_samples():
    mesh = M.icosphere(0.1, 2)
    sp = M.sampling_params(SimParams().set_particle_size(0.02), "R")
    a, _ = M.sample_surface(mesh, sp)
    sp.seed = 1234
    b, _ = M.sample_surface(mesh, sp)
    o, _ = oracle.sample_surface(mesh, sp)
    np.testing.assert_array_equal(b, o)
    assert len(a) != len(b) or not np.array_equal(a, b)


@pytest.mark.parametrize("field,value", [("minDistance", 0.0), ("maxDistance", 0.5), ("candidateMultiplier", 0)])
def test_gpu_sampler_rejects_invalid_parameters(field, value):
    sp = M.sampling_params(SimParams().set_particle_size(0.02), "R")
    setattr(sp, field, value)
    with pytest.raises(M.MeshError):
        M.sample_surface(M.icosphere(0.1, 1), sp)


def run_pair(st, dmin, dmax, p, steps):
    g, o = SimBackendB200(p), OracleBackend(p)
    for be in (g, o):
        be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)
        be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    for _ in range(steps):
        g.step(p)
        o.step(p)
    return g.push(), o.push()


def test_gpu_mesh_rigid_body_steps_like_oracle():
    st, dmin, dmax, p = S.floating_mesh_body()
    assert st.N_RB == 1 and st.N_R > 100
    a, b = run_pair(st, dmin, dmax, p, 10)
    for c in ("xCM", "yCM", "zCM"):
        assert abs(float(getattr(a, c)[0]) - float(getattr(b, c)[0])) <= 1e-5, c
    for c in ("xVelRB", "yVelRB", "zVelRB"):
        assert abs(float(getattr(a, c)[0]) - float(getattr(b, c)[0])) <= 1e-4, c
    np.testing.assert_array_equal(a.idF, b.idF)
    assert np.max(np.abs(a.yPosF - b.yPosF)) <= 1e-5


def test_gpu_mesh_boundary_obstacle_steps_like_oracle():
    st, dmin, dmax, p = S.floating_cubes()  # its fluid slab and tank, without the cubes
    base = UniversalSimState(st.N_F, st.N_B)
    for k in ["idF", "idB"] + FLUID_F32 + BOUNDARY_F32:
        setattr(base, k, getattr(st, k).copy())
    obst, stats = M.build_boundary_mesh(base, M.box_mesh((0.5, 0.5, 0.5)), p, 0.12, (0.45, 0.39, 0.3),
                                         M.euler_orientation(30.0, 0.0, 0.0))
    assert obst.N_B > st.N_B and stats.N_initialSamples > 0
    a, b = run_pair(obst, dmin, dmax, p, 5)
    np.testing.assert_array_equal(a.idF, b.idF)
    assert np.max(np.abs(a.xPosF - b.xPosF)) <= 1e-5
    np.testing.assert_allclose(np.sort(a.volB), np.sort(b.volB), rtol=1e-6)
