"""Mesh geometry for mesh boundaries / rigid bodies: the reference's known answers for uniform
scaling (tests/unit/triangle_surface.cpp) and rigid-body mass properties
(tests/unit/rigid_body_properties.cpp), the OBJ loading rules (obj_loading.cpp), and the
sampler's own guarantees checked on the oracle's restatement (minimum spacing, probe coverage,
determinism, the reference's parameter checks)."""
import math

import numpy as np
import pytest
from scipy.spatial import cKDTree

import oracle
from turbospharticles_b200 import mesh as M
from turbospharticles_b200.params import SimParams


def box():
    v = [(-1, -2, -3), (1, -2, -3), (1, 2, -3), (-1, 2, -3), (-1, -2, 3), (1, -2, 3), (1, 2, 3), (-1, 2, 3)]
    t = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (3, 7, 6), (3, 6, 2), (0, 4, 7), (0, 7, 3),
         (1, 2, 6), (1, 6, 5)]
    return M.TriangleSurfaceMesh(np.array(v, np.float32), np.array(t, np.uint32))


def tetra():
    v = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]
    t = [(0, 2, 1), (0, 1, 3), (0, 3, 2), (1, 2, 3)]
    return M.TriangleSurfaceMesh(np.array(v, np.float32), np.array(t, np.uint32))


TETRA_INV_INERTIA = np.array([[14, -2, -2], [-2, 14, -2], [-2, -2, 14]], np.float64)


def float_eq(a, b):
    """EXPECT_FLOAT_EQ: within 4 units in the last place of FP32."""
    a, b = np.float32(a), np.float32(b)
    return abs(int(a.view(np.int32)) - int(b.view(np.int32))) <= 4


def near_inv(actual, expected):
    assert np.all(np.abs(actual - expected) <= 1e-8 + 2e-6 * np.abs(expected)), (actual, expected)


# ---------------------------------------------------------------- ScaleToTargetExtent
def test_scales_uniformly_and_returns_scaled_box_center():
    m = M.TriangleSurfaceMesh(np.array([(-2, 1, -1), (6, 5, 3), (4, 2, 1)], np.float32), np.array([(0, 1, 2)]))
    c = M.scale_to_target_extent(m, 4.0)
    np.testing.assert_array_equal(m.vertices, np.array([(-1, 0.5, -0.5), (3, 2.5, 1.5), (2, 1, 0.5)], np.float32))
    np.testing.assert_array_equal(c, np.array([1.0, 1.5, 0.5], np.float32))
    np.testing.assert_array_equal(m.triangles, [[0, 1, 2]])


def test_accepts_planar_meshes():
    m = M.TriangleSurfaceMesh(np.array([(0, 0, 2), (2, 0, 2), (0, 4, 2)], np.float32), np.zeros((0, 3)))
    c = M.scale_to_target_extent(m, 8.0)
    assert (m.vertices[1, 0], m.vertices[2, 1], m.vertices[0, 2]) == (4.0, 8.0, 4.0)
    np.testing.assert_array_equal(c, np.array([2, 4, 4], np.float32))


def test_rejects_empty_and_zero_extent_meshes():
    with pytest.raises(M.MeshError):
        M.scale_to_target_extent(M.TriangleSurfaceMesh(np.zeros((0, 3)), np.zeros((0, 3))), 1.0)
    with pytest.raises(M.MeshError):
        M.scale_to_target_extent(M.TriangleSurfaceMesh(np.array([(1, 2, 3), (1, 2, 3)]), np.zeros((0, 3))), 1.0)


@pytest.mark.parametrize("target", [0.0, -1.0, math.inf, -math.inf, math.nan])
def test_rejects_invalid_target_extents(target):
    m = M.TriangleSurfaceMesh(np.array([(0, 0, 0), (1, 1, 1)], np.float32), np.zeros((0, 3)))
    with pytest.raises(M.MeshError):
        M.scale_to_target_extent(m, target)
    np.testing.assert_array_equal(m.vertices[1], [1, 1, 1])


# ---------------------------------------------------------------- RigidBodyPropertyComputer
def test_known_box_properties():
    p = M.rigid_body_properties(box(), 3.0)
    assert float_eq(p.volume, 48.0) and float_eq(p.mass, 144.0)
    assert np.max(np.abs(p.center_of_mass)) <= 1e-6
    near_inv(p.body_inertia_inv, np.diag([1 / 624.0, 1 / 480.0, 1 / 240.0]))


def test_known_tetrahedron_properties():
    p = M.rigid_body_properties(tetra(), 6.0)
    assert float_eq(p.volume, 1 / 6) and float_eq(p.mass, 1.0)
    assert np.max(np.abs(p.center_of_mass - 0.25)) <= 1e-6
    near_inv(p.body_inertia_inv, TETRA_INV_INERTIA)


def test_translation_moves_center_only():
    m = tetra()
    m.vertices += np.array([8, -4, 2], np.float32)
    p = M.rigid_body_properties(m, 6.0)
    assert float_eq(p.volume, 1 / 6) and float_eq(p.mass, 1.0)
    assert np.max(np.abs(p.center_of_mass - np.array([8.25, -3.75, 2.25]))) <= 1e-6
    near_inv(p.body_inertia_inv, TETRA_INV_INERTIA)


def test_rotation_rotates_center_and_inverse_inertia():
    m = box()
    x = m.vertices[:, 0] + np.float32(5)
    y = m.vertices[:, 1].copy()
    m.vertices[:, 0] = (np.float32(3) * x - np.float32(4) * y) / np.float32(5)
    m.vertices[:, 1] = (np.float32(4) * x + np.float32(3) * y) / np.float32(5)
    p = M.rigid_body_properties(m, 3.0)
    ix, iy = np.float32(1 / 624), np.float32(1 / 480)
    xy = np.float32(12) * (ix - iy) / np.float32(25)
    exp = np.array([[(9 * ix + 16 * iy) / 25, xy, 0], [xy, (16 * ix + 9 * iy) / 25, 0], [0, 0, 1 / 240]], np.float64)
    assert float_eq(p.volume, 48.0) and float_eq(p.mass, 144.0)
    assert np.max(np.abs(p.center_of_mass - np.array([3, 4, 0]))) <= 1e-6
    near_inv(p.body_inertia_inv, exp)


@pytest.mark.parametrize("scale", [0.5, 2.0])
def test_scales_with_mesh_size(scale):
    m = tetra()
    m.vertices *= np.float32(scale)
    p = M.rigid_body_properties(m, 6.0)
    assert float_eq(p.volume, scale ** 3 / 6) and float_eq(p.mass, scale ** 3)
    near_inv(p.body_inertia_inv, TETRA_INV_INERTIA / scale ** 5)


@pytest.mark.parametrize("density", [3.0, 6.0, 12.0])
def test_scales_with_density(density):
    p = M.rigid_body_properties(tetra(), density)
    assert float_eq(p.volume, 1 / 6) and float_eq(p.mass, density / 6)
    near_inv(p.body_inertia_inv, TETRA_INV_INERTIA * (6 / density))


def test_accepts_globally_reversed_winding():
    m = tetra()
    m.triangles = m.triangles[:, [0, 2, 1]].copy()
    p = M.rigid_body_properties(m, 6.0)
    assert float_eq(p.volume, 1 / 6) and float_eq(p.mass, 1.0)
    near_inv(p.body_inertia_inv, TETRA_INV_INERTIA)


def _bad_meshes():
    out = []
    m = tetra(); m.triangles = m.triangles[1:]; out.append(("open", m, 6.0))
    m = tetra(); m.triangles[0, [1, 2]] = m.triangles[0, [2, 1]]; out.append(("winding", m, 6.0))
    for a in range(3):
        m = tetra(); m.triangles[0, a] = 4; out.append((f"index{a}", m, 6.0))
        m = tetra(); m.triangles[0, a] = m.triangles[0, (a + 1) % 3]; out.append((f"repeat{a}", m, 6.0))
    m = tetra(); m.vertices[3] = (1, 1, 0); out.append(("zero volume", m, 6.0))
    m = tetra(); m.triangles = np.vstack([m.triangles, m.triangles[:1]]); out.append(("non-manifold edge", m, 6.0))
    m = tetra()
    v = np.vstack([m.vertices, np.array([(-1, 0, 0), (0, -1, 0), (0, 0, -1)], np.float32)])
    t2 = tetra().triangles.astype(np.int64)
    t2 = np.where(t2 != 0, t2 + 3, 0)[:, [0, 2, 1]]
    out.append(("disconnected fans", M.TriangleSurfaceMesh(v, np.vstack([m.triangles, t2])), 6.0))
    out.append(("empty", M.TriangleSurfaceMesh(np.zeros((0, 3)), np.zeros((0, 3))), 6.0))
    for d in (0.0, -1.0, math.inf, math.nan):
        out.append((f"density {d}", tetra(), d))
    return out


@pytest.mark.parametrize("name,mesh,density", _bad_meshes(), ids=lambda x: x if isinstance(x, str) else "")
def test_rejects_invalid_meshes(name, mesh, density):
    with pytest.raises(M.MeshError):
        M.rigid_body_properties(mesh, density)


# ---------------------------------------------------------------- OBJ loading
def test_obj_loader_fans_polygons_and_resolves_indices(tmp_path):
    (tmp_path / "m.obj").write_text("# comment\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvn 0 0 1\n"
                                    "f 1/1/1 2/2/1 3/3/1 4/4/1 # quad\nf -4 -2 -1\n")
    m = M.load_obj(str(tmp_path), "m.obj")
    np.testing.assert_array_equal(m.triangles, [[0, 1, 2], [0, 2, 3], [0, 2, 3]])
    assert m.vertices.shape == (4, 3)


@pytest.mark.parametrize("name,text", [("zero", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n"),
                                       ("range", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n"),
                                       ("short", "v 0 0 0\nv 1 0 0\nf 1 2\n"),
                                       ("vertex", "v 0 0\n"), ("nan", "v nan 0 0\n"),
                                       ("token", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 x\n"),
                                       ("empty", "# nothing\n")])
def test_obj_loader_rejects_invalid_files(tmp_path, name, text):
    (tmp_path / "m.obj").write_text(text)
    with pytest.raises(M.MeshError):
        M.load_obj(str(tmp_path), "m.obj")


@pytest.mark.parametrize("path", ["", "/abs/m.obj", "../m.obj", "m.stl", "missing.obj"])
def test_obj_loader_path_rules(tmp_path, path):
    with pytest.raises(M.MeshError):
        M.load_obj(str(tmp_path), path)


# ---------------------------------------------------------------- sampler (oracle restatement)
def params(h=0.02):
    return SimParams().set_particle_size(h)


@pytest.mark.parametrize("name,mesh", [("sphere", M.icosphere(0.1, 2)), ("box", M.box_mesh((0.1, 0.06, 0.04))),
                                       ("tetra", tetra())])
def test_oracle_sampler_spacing_and_coverage(name, mesh):
    if name == "tetra":
        mesh = mesh.copy()
        M.scale_to_target_extent(mesh, 0.15)
    sp = M.sampling_params(params(), "R")
    s, st = oracle.sample_surface(mesh, sp)
    assert len(s) == st.N_initialSamples + st.N_coverageRepairs > 0
    d, _ = cKDTree(s.astype(np.float64)).query(s.astype(np.float64), k=2)
    assert d[:, 1].min() >= sp.minDistance * (1 - 1e-6)
    # every lattice probe is within the coverage target of a sample
    target = max(sp.minDistance, sp.maxDistance - sp.coverageProbeSpacing)
    probes = []
    for a, b, c in mesh.triangles:
        v0, v1, v2 = mesh.vertices[a], mesh.vertices[b], mesh.vertices[c]
        e = max(np.linalg.norm(v1 - v0), np.linalg.norm(v2 - v1), np.linalg.norm(v0 - v2))
        n = max(1, math.ceil(np.float32(e) / np.float32(sp.coverageProbeSpacing)))
        for i in range(n + 1):
            for j in range(n + 1 - i):
                probes.append((v0 * i + v1 * j + v2 * (n - i - j)) / n)
    assert len(probes) == st.N_coverageProbes
    dp, _ = cKDTree(s.astype(np.float64)).query(np.array(probes, np.float64))
    assert dp.max() <= target * (1 + 1e-4)


def test_oracle_sampler_is_deterministic_and_seeded():
    mesh = M.icosphere(0.1, 2)
    sp = M.sampling_params(params(), "R")
    a, _ = oracle.sample_surface(mesh, sp)
    b, _ = oracle.sample_surface(mesh, sp)
    np.testing.assert_array_equal(a, b)
    sp.seed = 7
    c, _ = oracle.sample_surface(mesh, sp)
    assert len(c) != len(a) or not np.array_equal(a, c)


@pytest.mark.parametrize("field,value", [("minDistance", 0.0), ("maxDistance", 0.5), ("coverageProbeSpacing", 0.0),
                                         ("candidateMultiplier", 0), ("maxDistance", 0.017)])
def test_oracle_sampler_rejects_invalid_parameters(field, value):
    sp = M.sampling_params(params(), "R")
    setattr(sp, field, value)
    with pytest.raises(M.MeshError):
        oracle.sample_surface(M.icosphere(0.1, 1), sp)
