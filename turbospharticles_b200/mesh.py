"""Triangle meshes for mesh boundaries and mesh rigid bodies: OBJ loading, uniform scaling,
rigid-body mass properties, GPU surface sampling, and the scene builders that turn a sampled
surface into boundary particles or a rigid body.

Follows the reference's scene geometry (source/simulation/scene/geometry/obj_loading.cpp,
triangle_surface.cpp, rigid_body_properties.cpp, surface_sampling.cpp) and builders
(scene/builder.cpp:1089-1260 BuildRigidBody_FromSurfaceSamples / BuildBoundary_FromSurfaceSamples,
rigid_mesh_helpers.h, boundary_mesh_helpers.h). Mesh errors raise MeshError with the
reference's messages.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

from . import abi
from .abi import TspError


class MeshError(RuntimeError):
    """A mesh the reference's loader, property computer or sampler rejects."""


@dataclass
class TriangleSurfaceMesh:
    """Scene::TriangleSurfaceMesh (triangle_surface.h): float32 (N, 3) vertices, uint32 (M, 3)
    triangles."""
    vertices: np.ndarray
    triangles: np.ndarray

    def __post_init__(self):
        self.vertices = np.ascontiguousarray(np.asarray(self.vertices, np.float32).reshape(-1, 3))
        self.triangles = np.ascontiguousarray(np.asarray(self.triangles, np.uint32).reshape(-1, 3))

    def copy(self) -> "TriangleSurfaceMesh":
        return TriangleSurfaceMesh(self.vertices.copy(), self.triangles.copy())


def load_obj(model_directory: str, model_file: str) -> TriangleSurfaceMesh:
    """ObjMeshLoader::Load (obj_loading.cpp:25-158): relative `.obj` path inside the model
    directory, `v x y z` vertices, `f` faces with 1-based or negative indices (texture / normal
    parts after '/' ignored), polygons triangulated as a fan from the first vertex."""
    if not model_file or os.path.isabs(model_file):
        raise MeshError("Rigid mesh model file must be a non-empty relative path.")
    if ".." in model_file.replace("\\", "/").split("/"):
        raise MeshError("Rigid mesh model file must remain inside the model directory.")
    if os.path.splitext(model_file)[1] != ".obj":
        raise MeshError("Rigid mesh model file must use the .obj extension.")
    path = os.path.normpath(os.path.join(model_directory, os.path.normpath(model_file)))
    try:
        lines = open(path, encoding="utf-8", errors="replace").read().splitlines()
    except OSError:
        raise MeshError(f"Could not open rigid mesh model file '{path}'.") from None
    verts, tris = [], []
    for no, line in enumerate(lines, 1):
        tok = line.split()
        if not tok or tok[0].startswith("#"):
            continue
        if tok[0] == "v":
            try:
                v = [np.float32(float(t)) for t in tok[1:4]]
            except ValueError:
                v = []
            if len(v) != 3 or not all(math.isfinite(x) for x in v):
                raise MeshError(f"Rigid mesh OBJ contains an invalid vertex at line {no}.")
            verts.append(v)
            continue
        if tok[0] != "f":
            continue
        face = []
        for t in tok[1:]:
            if t.startswith("#"):
                break
            it = t.split("/")[0]
            if not it:
                raise MeshError(f"Rigid mesh OBJ contains an invalid face at line {no}.")
            try:
                k = int(it)
            except ValueError:
                raise MeshError(f"Rigid mesh OBJ contains an invalid face index at line {no}.") from None
            if k == 0:
                raise MeshError(f"Rigid mesh OBJ contains a zero face index at line {no}.")
            idx = k - 1 if k > 0 else len(verts) + k
            if idx < 0 or idx >= len(verts):
                raise MeshError(f"Rigid mesh OBJ face index is out of range at line {no}.")
            face.append(idx)
        if len(face) < 3:
            raise MeshError(f"Rigid mesh OBJ contains a face with fewer than three vertices at line {no}.")
        tris.extend([face[0], face[i], face[i + 1]] for i in range(1, len(face) - 1))
    if not verts or not tris:
        raise MeshError("Rigid mesh OBJ does not contain a triangle surface.")
    return TriangleSurfaceMesh(np.array(verts, np.float32), np.array(tris, np.uint32))


def scale_to_target_extent(mesh: TriangleSurfaceMesh, target_extent: float) -> np.ndarray:
    """ScaleToTargetExtent (triangle_surface.cpp:13-61): scale uniformly so the largest
    bounding-box extent equals `target_extent`; returns the scaled box centre (FP32)."""
    f32 = np.float32
    t = f32(target_extent)
    if not math.isfinite(t) or t <= 0:
        raise MeshError("Mesh model target extent must be > 0.")
    if mesh.vertices.size == 0:
        raise MeshError("Cannot scale an empty triangle surface.")
    mn, mx = mesh.vertices.min(axis=0), mesh.vertices.max(axis=0)
    ext = mx - mn
    raw = f32(max(ext[0], max(ext[1], ext[2])))
    if not math.isfinite(raw) or raw <= 0:
        raise MeshError("Mesh model extent must be > 0.")
    with np.errstate(over="ignore", invalid="ignore"):
        s = f32(t / raw)
    if not math.isfinite(s) or s <= 0:
        raise MeshError("Mesh model scale must be > 0.")
    mesh.vertices *= s
    return (f32(0.5) * (mn + mx)) * s


@dataclass
class RigidBodyPhysicalProperties:
    center_of_mass: np.ndarray   # float32 (3,)
    body_inertia_inv: np.ndarray  # float32 (3, 3), row = first index
    volume: float
    mass: float


def rigid_body_properties(mesh: TriangleSurfaceMesh, density: float) -> RigidBodyPhysicalProperties:
    """RigidBodyPropertyComputer::Compute (rigid_body_properties.cpp:103-316): closed,
    consistently oriented, vertex-manifold surface required; signed tetrahedra moments in FP64
    (volume, first and second moments about the origin), shifted to the centre of mass; inertia
    inverted in FP64 and returned in FP32."""
    V, Tr = mesh.vertices, mesh.triangles
    if V.size == 0 or Tr.size == 0:
        raise MeshError("Rigid mesh does not contain a triangle surface.")
    if not math.isfinite(density) or density <= 0:
        raise MeshError("Rigid body density must be > 0.")
    if not np.all(np.isfinite(V)):
        raise MeshError("Rigid mesh contains a non-finite vertex.")
    nV = len(V)
    edges: dict = {}
    incident = [[] for _ in range(nV)]
    for t, (a, b, c) in enumerate(Tr.tolist()):
        if a >= nV or b >= nV or c >= nV:
            raise MeshError("Rigid mesh contains an invalid vertex index.")
        if a == b or a == c or b == c:
            raise MeshError("Rigid mesh contains a degenerate triangle.")
        for u, v in ((a, b), (b, c), (c, a)):
            key = (u, v) if u < v else (v, u)
            e = edges.setdefault(key, [0, 0, []])
            if e[0] < 2:
                e[2].append(t)
            e[0] += 1
            e[1] += 1 if u < v else -1
            if e[0] > 2:
                raise MeshError("Rigid mesh contains an edge shared by more than two triangles.")
        for u in (a, b, c):
            incident[u].append(t)
    nbr = [[] for _ in range(len(Tr))]
    for n, orient, ts in edges.values():
        if n != 2 or orient != 0:
            raise MeshError("Rigid mesh must be a closed consistently oriented triangle surface.")
        nbr[ts[0]].append(ts[1])
        nbr[ts[1]].append(ts[0])
    for inc in incident:  # one connected triangle fan per vertex
        if not inc:
            continue
        inc_set, seen, pending = set(inc), set(), [inc[0]]
        while pending:
            t = pending.pop()
            if t in seen:
                continue
            seen.add(t)
            pending.extend(n for n in nbr[t] if n in inc_set)
        if len(seen) != len(inc):
            raise MeshError("Rigid mesh is non-manifold at a vertex.")
    vol, first, second = 0.0, np.zeros(3), np.zeros((3, 3))
    Vd = V.astype(np.float64)
    for a, b, c in Tr.tolist():
        pa, pb, pc = Vd[a], Vd[b], Vd[c]
        tv = float(np.dot(pa, np.cross(pb, pc))) / 6.0
        if not math.isfinite(tv):
            raise MeshError("Rigid mesh volume computation is not finite.")
        vol += tv
        first += tv * (pa + pb + pc) / 4.0
        second += tv * (0.1 * (np.outer(pa, pa) + np.outer(pb, pb) + np.outer(pc, pc))
                        + 0.05 * (np.outer(pa, pb) + np.outer(pb, pa) + np.outer(pa, pc) + np.outer(pc, pa)
                                  + np.outer(pb, pc) + np.outer(pc, pb)))
    if (not math.isfinite(vol) or not np.all(np.isfinite(first)) or not np.all(np.isfinite(second))
            or abs(vol) <= np.finfo(np.float64).eps):
        raise MeshError("Rigid mesh enclosed volume is invalid.")
    if vol < 0:
        vol, first, second = -vol, -first, -second
    com = first / vol
    central = second - vol * np.outer(com, com)
    inertia = (np.eye(3) * np.trace(central) - central) * float(density)
    mass = vol * float(density)
    det = float(np.linalg.det(inertia))
    f32max = float(np.finfo(np.float32).max)
    if (not math.isfinite(mass) or not np.all(np.isfinite(inertia)) or not math.isfinite(det) or mass > f32max
            or vol > f32max or det <= 0 or min(inertia[0, 0], inertia[1, 1], inertia[2, 2]) <= 0):
        raise MeshError("Rigid mesh physical properties are invalid.")
    inv = np.linalg.inv(inertia)
    if not np.all(np.isfinite(inv)):
        raise MeshError("Rigid mesh inverse inertia is not finite.")
    with np.errstate(over="ignore"):
        props = RigidBodyPhysicalProperties(com.astype(np.float32), inv.astype(np.float32), float(np.float32(vol)),
                                            float(np.float32(mass)))
    if (not math.isfinite(props.volume) or props.volume <= 0 or not math.isfinite(props.mass) or props.mass <= 0
            or not np.all(np.isfinite(props.center_of_mass)) or not np.all(np.isfinite(props.body_inertia_inv))):
        raise MeshError("Rigid mesh physical properties exceed float limits.")
    return props


# ---------------------------------------------------------------------------- simple solids
def box_mesh(half=(0.5, 0.5, 0.5)) -> TriangleSurfaceMesh:
    """Closed, outward-wound box of half extents `half` around the origin."""
    hx, hy, hz = half
    v = [(-hx, -hy, -hz), (hx, -hy, -hz), (hx, hy, -hz), (-hx, hy, -hz),
         (-hx, -hy, hz), (hx, -hy, hz), (hx, hy, hz), (-hx, hy, hz)]
    t = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4),
         (3, 7, 6), (3, 6, 2), (0, 4, 7), (0, 7, 3), (1, 2, 6), (1, 6, 5)]
    return TriangleSurfaceMesh(np.array(v, np.float32), np.array(t, np.uint32))


def icosphere(radius=0.5, subdivisions=2) -> TriangleSurfaceMesh:
    """Closed, outward-wound icosahedral sphere (a curved, non-axis-aligned test surface)."""
    p = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
         (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    v = [np.array(x, np.float64) / np.linalg.norm(x) for x in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        cache, nf = {}, []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return TriangleSurfaceMesh((np.array(v) * radius).astype(np.float32), np.array(f, np.uint32))


# ---------------------------------------------------------------------------- sampling
def sampling_params(params, kind: str = "R"):
    """tsp_surface_sampling_params from SimParams (parameters_sim.h:122-139): distances of the
    boundary ("B") or rigid ("R") sampler."""
    sp = abi.TspSurfaceSamplingParams()
    sp.minDistance = getattr(params, f"surfaceSamplingMinDistance{kind}")
    sp.maxDistance = getattr(params, f"surfaceSamplingMaxDistance{kind}")
    sp.coverageProbeSpacing = getattr(params, f"surfaceSamplingCoverageProbeSpacing{kind}")
    sp.particleSizeF = params.particleSizeF
    sp.candidateMultiplier = params.surfaceSamplingCandidateMultiplier
    sp.seed = params.surfaceSamplingSeed
    return sp


def _sample_with(fn, mesh: TriangleSurfaceMesh, sp, err):
    v, t = mesh.vertices, mesh.triangles
    est = 0
    if len(t) and sp.minDistance > 0 and np.all(t < len(v)) and np.all(np.isfinite(v)):
        area = 0.5 * float(np.sum(np.linalg.norm(np.cross(v[t[:, 1]].astype(np.float64) - v[t[:, 0]],
                                                          v[t[:, 2]].astype(np.float64) - v[t[:, 0]]), axis=1)))
        est = int(min(area / (sp.minDistance * sp.minDistance), 1e8))
    cap = 2 * est + 1024
    stats = abi.TspSurfaceSamplingStats()
    for _ in range(2):
        out = np.zeros((cap, 3), np.float32)
        n = C.c_uint64()
        rc = fn(v.ctypes.data_as(C.POINTER(C.c_float)), len(v), t.ctypes.data_as(C.POINTER(C.c_uint32)), len(t),
                C.byref(sp), out.ctypes.data_as(C.POINTER(C.c_float)), cap, C.byref(n), C.byref(stats))
        if rc == abi.TSP_ERR_OVERFLOW:
            cap = n.value
            continue
        if rc == abi.TSP_ERR_INVALID:
            raise MeshError(err())
        if rc != 0:
            raise TspError(rc, err())
        return out[:n.value].copy(), stats
    raise MeshError("surface sample count changed between two identical calls")


def sample_surface(mesh: TriangleSurfaceMesh, sp, device: int = -1):
    """SurfaceSampler::Sample on the GPU (tsp_b200_sample_surface): (N, 3) float32 samples and
    the sampling statistics."""
    L = abi.load_library()
    return _sample_with(lambda *a: L.tsp_b200_sample_surface(device, *a), mesh, sp,
                        lambda: L.tsp_b200_last_error(None).decode())


# ---------------------------------------------------------------------------- scene builders
def euler_orientation(yaw_deg=0.0, pitch_deg=0.0, roll_deg=0.0) -> np.ndarray:
    """Turn around world Y, then tilt around local Z (pitch) and local X (roll)."""
    def rot(axis, deg):
        c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
        if axis == "x":
            return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
        if axis == "y":
            return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
        return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])
    return (rot("y", yaw_deg) @ rot("z", pitch_deg) @ rot("x", roll_deg)).astype(np.float32)


def append_rigid_body(st, samples_local: np.ndarray, com, orientation, mass: float, body_inertia_inv,
                      init_vel=(0.0, 0.0, 0.0), init_omega=(0.0, 0.0, 0.0), params=None):
    """BuildRigidBody_FromSurfaceSamples (builder.cpp:1089-1205) + ApplyInitialRigidBodyState
    (rigid_mesh_helpers.h): append one body with its body-frame surface samples to a
    UniversalSimState; returns the new state (arrays grow, existing particles keep their order)."""
    from .state import BODY_F32, RIGID_F32, UniversalSimState
    n_add = len(samples_local)
    out = UniversalSimState(st.N_F, st.N_B, st.N_R + n_add, st.N_RB + 1)
    for k, v in st.__dict__.items():
        if not isinstance(v, np.ndarray):
            if k not in ("N_F", "N_B", "N_R", "N_RB"):
                setattr(out, k, v)
        elif k in ("idR", "bodyIdR") or k in RIGID_F32:
            getattr(out, k)[:st.N_R] = v
        elif k in ("idRB", "rigidParticleCountRB") or k in BODY_F32:
            getattr(out, k)[:st.N_RB] = v
        else:
            setattr(out, k, v.copy())
    b, r0 = st.N_RB, st.N_R
    A = np.asarray(orientation, np.float32)
    out.idRB[b] = b
    out.rigidParticleCountRB[b] = n_add
    out.xCM[b], out.yCM[b], out.zCM[b] = np.asarray(com, np.float32)
    for i in range(3):
        for j in range(3):
            getattr(out, f"a{i}{j}")[b] = A[i, j]
            getattr(out, f"iBodyInv{i}{j}")[b] = np.float32(body_inertia_inv[i, j])
    out.massRB[b] = np.float32(mass)
    out.massInvRB[b] = np.float32(1.0) / np.float32(mass) if mass > 0 else 0.0
    out.idR[r0:] = (np.uint64(st.N_R) + np.arange(n_add, dtype=np.uint64)) if st.N_R else np.arange(n_add, dtype=np.uint64)
    out.bodyIdR[r0:] = b
    out.xPosRelR[r0:], out.yPosRelR[r0:], out.zPosRelR[r0:] = (samples_local[:, k] for k in range(3))
    if params is not None:  # default coefficients until the volume stage runs (state_sim.h:461-475)
        out.psiR[r0:] = np.float32(params.massB)
        out.volR[r0:] = np.float32(np.float32(params.massB) / np.float32(params.restDensity))
    out.xVelRB[b], out.yVelRB[b], out.zVelRB[b] = init_vel
    out.xOmegaRB[b], out.yOmegaRB[b], out.zOmegaRB[b] = init_omega
    w_body = A.T.astype(np.float64) @ np.asarray(init_omega, np.float64)
    L_world = A.astype(np.float64) @ (np.linalg.inv(np.asarray(body_inertia_inv, np.float64)) @ w_body)
    out.xAngMomRB[b], out.yAngMomRB[b], out.zAngMomRB[b] = L_world.astype(np.float32)
    return out


def build_rigid_mesh(st, mesh: TriangleSurfaceMesh, params, target_extent: float, density: float, center,
                     orientation=None, init_vel=(0.0, 0.0, 0.0), init_omega=(0.0, 0.0, 0.0), sampler=None):
    """BuildRigidMesh (rigid_mesh_helpers.h): scale the model, compute its mass properties, move
    it into its centre-of-mass frame, sample its surface (GPU sampler by default) and append the
    body at `center`. Returns (new state, sampling stats)."""
    m = mesh.copy()
    scale_to_target_extent(m, target_extent)
    props = rigid_body_properties(m, density)
    m.vertices -= props.center_of_mass
    samples, stats = (sampler or sample_surface)(m, sampling_params(params, "R"))
    A = euler_orientation() if orientation is None else np.asarray(orientation, np.float32)
    return append_rigid_body(st, samples, center, A, props.mass, props.body_inertia_inv, init_vel, init_omega,
                             params), stats


def build_boundary_mesh(st, mesh: TriangleSurfaceMesh, params, target_extent: float, center, orientation=None,
                        sampler=None):
    """BuildBoundaryMesh (boundary_mesh_helpers.h): scale the model about its box centre, sample
    its surface and append the samples, posed at `center`, as boundary particles (volumes and
    psi from the boundary-volume stage). Returns (new state, sampling stats)."""
    from .state import BOUNDARY_F32, UniversalSimState
    m = mesh.copy()
    c = scale_to_target_extent(m, target_extent)
    m.vertices -= c
    samples, stats = (sampler or sample_surface)(m, sampling_params(params, "B"))
    A = euler_orientation() if orientation is None else np.asarray(orientation, np.float32)
    world = (samples.astype(np.float32) @ A.T + np.asarray(center, np.float32)).astype(np.float32)
    n_add = len(world)
    out = UniversalSimState(st.N_F, st.N_B + n_add, st.N_R, st.N_RB)
    for k, v in st.__dict__.items():
        if not isinstance(v, np.ndarray):
            if k not in ("N_F", "N_B", "N_R", "N_RB"):
                setattr(out, k, v)
        elif k == "idB" or k in BOUNDARY_F32:
            getattr(out, k)[:st.N_B] = v
        else:
            setattr(out, k, v.copy())
    out.idB[st.N_B:] = np.uint64(st.N_B) + np.arange(n_add, dtype=np.uint64)
    out.xPosB[st.N_B:], out.yPosB[st.N_B:], out.zPosB[st.N_B:] = world[:, 0], world[:, 1], world[:, 2]
    out.psiB[st.N_B:] = np.float32(params.massB)  # defaults until the volume stage runs (state_sim.h:347-362)
    out.volB[st.N_B:] = np.float32(np.float32(params.massB) / np.float32(params.restDensity))
    return out, stats
