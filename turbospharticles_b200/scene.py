"""Seeded synthetic scenes for the IISPH step.

Restates the reference scene builder in FP32 numpy so generated particles are identical to
the reference's:
  - TilesCount / StartOffset / Jitter3D ............ source/simulation/scene/builder.cpp:1485-1525
  - BuildFluidBlock_OBB ............................ builder.cpp:455-642
  - BuildBoundaryContainer_OBB + layers on faces ... builder.cpp:415-453, 1354-1372, 1400-1483
  - BuildRigidBody_OBB_Hollow ...................... builder.cpp:925-1087, 1527-1540
  - ComputeSimDomainBounds ......................... source/simulation/scene/scenario_sim.cpp:123-148
Boundary/rigid volumes (builder.cpp:174-376) are computed by the backend stage
`STAGE_BOUNDARY_VOLUMES` on the GPU, not here.

Neighbor-search-only inputs (uniform / Gaussian-clustered points in the unit cube) have no
counterpart in the reference builder; they are seeded numpy draws with the workload's sizes.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .params import SimParams
from .state import UniversalSimState

f32 = np.float32


@dataclasses.dataclass
class OBB:
    origin: tuple
    lengths: tuple  # (uLen, vLen, wLen)
    u: tuple = (1.0, 0.0, 0.0)
    v: tuple = (0.0, 1.0, 0.0)
    w: tuple = (0.0, 0.0, 1.0)


def _v(t):
    return np.asarray(t, dtype=f32)


def tiles_count(length, spacing) -> int:
    """builder.cpp:1511-1525 (floor(length / spacing) + 1 in FP32, at least 1)."""
    if spacing <= 0:
        return 0
    intervals = math.floor(float(f32(f32(length) / f32(spacing))))
    return max(1, int(intervals + 1))


def start_offset(length, spacing, n) -> float:
    """builder.cpp:1503-1509."""
    if n <= 1:
        return f32(0.0)
    covered = f32(f32(n - 1) * f32(spacing))
    return f32(f32(0.5) * max(f32(0.0), f32(f32(length) - covered)))


def jitter3d(base_seed: int, key: np.ndarray, amp: float) -> np.ndarray:
    """SplitMix64-style hash jitter (builder.cpp:1486-1501), vectorised over keys."""
    with np.errstate(over="ignore"):
        x = np.uint64(base_seed & 0xFFFFFFFFFFFFFFFF) + key.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        x ^= x >> np.uint64(30)
        x *= np.uint64(0xBF58476D1CE4E5B9)
        x ^= x >> np.uint64(27)
        x *= np.uint64(0x94D049BB133111EB)
        x ^= x >> np.uint64(31)
    u01 = (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return ((u01 * 2.0 - 1.0) * float(f32(amp))).astype(f32)


def _combine(origin, axes, coords):
    """origin + a0*c0 + a1*c1 + a2*c2 with glm's left-to-right FP32 evaluation."""
    out = []
    for comp in range(3):
        acc = np.full(coords[0].shape, origin[comp], dtype=f32)
        for a, c in zip(axes, coords):
            acc = (acc + (f32(a[comp]) * c).astype(f32)).astype(f32)
        out.append(acc)
    return out


def fluid_block(box: OBB, p: SimParams, id_base: int = 0):
    """BuildFluidBlock_OBB without a build region: returns ids and FP32 x, y, z."""
    size = f32(p.particleSizeF)
    radius = f32(size * f32(0.5))
    L = [f32(x) for x in box.lengths]
    Li = [f32(l - f32(f32(2.0) * radius)) for l in L]
    if min(Li) <= 0:
        return np.zeros(0, np.uint64), *(np.zeros(0, f32) for _ in range(3))
    N = [tiles_count(l, size) for l in Li]
    off = [f32(radius + start_offset(Li[a], size, N[a])) for a in range(3)]
    jit = f32(f32(p.jitterFracF) * f32(p.particleSizeF))
    kw, jv, iu = np.meshgrid(np.arange(N[2]), np.arange(N[1]), np.arange(N[0]), indexing="ij")
    kw, jv, iu = kw.ravel(), jv.ravel(), iu.ravel()
    idx = (np.uint64(id_base) + ((kw.astype(np.uint64) * np.uint64(N[1]) + jv.astype(np.uint64))
                                 * np.uint64(N[0]) + iu.astype(np.uint64)))
    u = (off[0] + (iu.astype(f32) * size)).astype(f32)
    v = (off[1] + (jv.astype(f32) * size)).astype(f32)
    w = (off[2] + (kw.astype(f32) * size)).astype(f32)
    if jit > 0:
        seed = int(p.jitterSeedF) & 0xFFFFFFFFFFFFFFFF
        k3 = idx * np.uint64(3)
        u = (u + jitter3d(seed, k3, jit)).astype(f32)
        v = (v + jitter3d(seed, k3 + np.uint64(1), jit)).astype(f32)
        w = (w + jitter3d(seed, k3 + np.uint64(2), jit)).astype(f32)
    u = np.clip(u, radius, f32(L[0] - radius)).astype(f32)
    v = np.clip(v, radius, f32(L[1] - radius)).astype(f32)
    w = np.clip(w, radius, f32(L[2] - radius)).astype(f32)
    x, y, z = _combine(_v(box.origin), (_v(box.u), _v(box.v), _v(box.w)), (u, v, w))
    return idx, x, y, z


def _faces(box: OBB):
    """GetFacesFromOBB (builder.cpp:1354-1372): (origin, uHat, vHat, nHat, uLen, vLen)."""
    o, u, v, w = _v(box.origin), _v(box.u), _v(box.v), _v(box.w)
    uL, vL, wL = (f32(x) for x in box.lengths)
    return [
        [o, u, v, -w, uL, vL],
        [(o + (w * wL).astype(f32)).astype(f32), u, v, w, uL, vL],
        [o, w, v, -u, wL, vL],
        [(o + (u * uL).astype(f32)).astype(f32), w, v, u, wL, vL],
        [o, u, w, -v, uL, wL],
        [(o + (v * vL).astype(f32)).astype(f32), u, w, v, uL, wL],
    ]


def boundary_container(box: OBB, p: SimParams, id_base: int = 0):
    """BuildBoundaryContainer_OBB (builder.cpp:415-453) without the coefficient pass."""
    if p.boundaryLayers <= 0:
        return np.zeros(0, np.uint64), *(np.zeros(0, f32) for _ in range(3))
    size = f32(p.particleSizeB)
    radius = f32(size * f32(0.5))
    pad = f32(radius + f32(f32(f32(p.boundaryLayers) - f32(1.0)) * size))
    faces = _faces(box)

    def extend(f, pu, pv):
        o, uh, vh, nh, uL, vL = f
        shift = ((uh * f32(pu)).astype(f32) + (vh * f32(pv)).astype(f32)).astype(f32)
        return [(o - shift).astype(f32), uh, vh, nh, f32(uL + f32(f32(2.0) * f32(pu))),
                f32(vL + f32(f32(2.0) * f32(pv)))]

    faces[2] = extend(faces[2], pad, pad)
    faces[3] = extend(faces[3], pad, pad)
    faces[4] = extend(faces[4], 0.0, pad)
    faces[5] = extend(faces[5], 0.0, pad)
    ids, xs, ys, zs = [], [], [], []
    base = id_base
    for o, uh, vh, nh, uL, vL in faces:
        Nu, Nv = tiles_count(uL, size), tiles_count(vL, size)
        layer, i, j = np.meshgrid(np.arange(p.boundaryLayers), np.arange(Nu), np.arange(Nv),
                                  indexing="ij")
        layer, i, j = layer.ravel(), i.ravel(), j.ravel()
        su = np.minimum((i.astype(f32) * size).astype(f32), uL).astype(f32)
        sv = np.minimum((j.astype(f32) * size).astype(f32), vL).astype(f32)
        out = (f32(size * f32(0.5)) + (layer.astype(f32) * size).astype(f32)).astype(f32)
        comps = []
        for c in range(3):
            acc = np.full(su.shape, o[c], f32)
            acc = (acc + (f32(uh[c]) * su).astype(f32)).astype(f32)
            acc = (acc + (f32(vh[c]) * sv).astype(f32)).astype(f32)
            acc = (acc + (f32(nh[c]) * out).astype(f32)).astype(f32)
            comps.append(acc)
        n_face = p.boundaryLayers * Nu * Nv
        ids.append(np.uint64(base) + ((layer.astype(np.uint64) * np.uint64(Nu) + i.astype(np.uint64))
                                      * np.uint64(Nv) + j.astype(np.uint64)))
        base += n_face
        xs.append(comps[0]); ys.append(comps[1]); zs.append(comps[2])
    return (np.concatenate(ids), np.concatenate(xs), np.concatenate(ys), np.concatenate(zs))


def sim_domain_bounds(boxes, p: SimParams):
    """ComputeSimDomainBounds (scenario_sim.cpp:123-148) for axis-aligned boxes."""
    mn = np.array(boxes[0].origin, f32)
    mx = np.array(boxes[0].origin, f32)
    for b in boxes:
        o = np.array(b.origin, f32)
        e = (o + np.array(b.lengths, f32)).astype(f32)
        mn = np.minimum(mn, np.minimum(o, e))
        mx = np.maximum(mx, np.maximum(o, e))
    pad = f32((f32(p.boundaryLayers) - f32(0.5)) * f32(p.particleSizeB)) if p.boundaryLayers > 0 else f32(0)
    return (mn - pad).astype(f32), (mx + pad).astype(f32)


def hollow_box_count(Nu, Nv, Nw, layers):
    lw = 2 * layers
    inner = max(Nu - lw, 0) * max(Nv - lw, 0) * max(Nw - lw, 0)
    return Nu * Nv * Nw - inner


def rigid_hollow_box(box: OBB, p: SimParams, density: float):
    """BuildRigidBody_OBB_Hollow (builder.cpp:925-1087) without jitter: body-frame particle
    positions and body properties (mass, diagonal inverse inertia, orientation = box axes)."""
    size = f32(p.particleSizeB)
    radius = f32(size * f32(0.5))
    L = [f32(x) for x in box.lengths]
    Li = [f32(l - f32(f32(2.0) * radius)) for l in L]
    N = [tiles_count(l, size) for l in Li]
    u_, v_, w_ = _v(box.u), _v(box.v), _v(box.w)
    o = _v(box.origin)
    origin_i = (((o + (u_ * radius).astype(f32)).astype(f32) + (v_ * radius).astype(f32)).astype(f32)
                + (w_ * radius).astype(f32)).astype(f32)
    layers = p.boundaryLayers
    kw, jv, iu = np.meshgrid(np.arange(N[2]), np.arange(N[1]), np.arange(N[0]), indexing="ij")
    kw, jv, iu = kw.ravel(), jv.ravel(), iu.ravel()
    inside = ((iu >= layers) & (iu <= N[0] - 1 - layers) & (jv >= layers) & (jv <= N[1] - 1 - layers)
              & (kw >= layers) & (kw <= N[2] - 1 - layers))
    keep = ~inside
    iu, jv, kw = iu[keep], jv[keep], kw[keep]
    uu = np.minimum(Li[0], (iu.astype(f32) * size).astype(f32)).astype(f32)
    vv = np.minimum(Li[1], (jv.astype(f32) * size).astype(f32)).astype(f32)
    ww = np.minimum(Li[2], (kw.astype(f32) * size).astype(f32)).astype(f32)
    pos = _combine(origin_i, (u_, v_, w_), (uu, vv, ww))
    half = [f32(f32(0.5) * l) for l in L]
    center = [c[0] for c in _combine(o, (u_, v_, w_), tuple(np.array([h], f32) for h in half))]
    rel = [(pos[c] - center[c]).astype(f32) for c in range(3)]

    def dot(a):
        return ((rel[0] * a[0]).astype(f32) + (rel[1] * a[1]).astype(f32) + (rel[2] * a[2]).astype(f32)).astype(f32)

    local = (dot(u_), dot(v_), dot(w_))
    vol = f32(f32(L[0] * L[1]) * L[2])
    mass = f32(f32(density) * vol) if density > 0 else f32(0)
    mass_inv = f32(f32(1.0) / mass) if mass > 0 else f32(0)

    def iinv(a, b):
        return f32(f32(12.0) / f32(mass * f32(f32(a * a) + f32(b * b)))) if mass > 0 else f32(0)

    body = dict(center=center, mass=mass, massInv=mass_inv,
                iBodyInv=(iinv(L[1], L[2]), iinv(L[0], L[2]), iinv(L[0], L[1])),
                A=np.array([[u_[0], v_[0], w_[0]], [u_[1], v_[1], w_[1]], [u_[2], v_[2], w_[2]]], f32))
    return local, body


# ----------------------------------------------------------------------------------- scenes

def breaking_dam(container: OBB, fluid: OBB, p: SimParams, rigid=None):
    """BreakingDamScene::Build (source/simulation/scene/scenarios/breaking_dam.h:40-45):
    container walls first, then the fluid block (or a list of blocks, IDs consecutive);
    optional hollow rigid boxes
    [(OBB, density), ...]. Returns (state, domain_min, domain_max)."""
    idB, xB, yB, zB = boundary_container(container, p)
    parts, base = [], 0
    for box in (fluid if isinstance(fluid, (list, tuple)) else [fluid]):
        parts.append(fluid_block(box, p, id_base=base))
        base += parts[-1][0].shape[0]
    idF, xF, yF, zF = (np.concatenate([q[c] for q in parts]) for c in range(4))
    bodies = []
    rel = [[], [], []]
    body_of = []
    for k, (box, dens) in enumerate(rigid or []):
        local, body = rigid_hollow_box(box, p, dens)
        for c in range(3):
            rel[c].append(local[c])
        body_of.append(np.full(local[0].shape[0], k, np.uint32))
        bodies.append(body)
    N_R = int(sum(r.shape[0] for r in rel[0]))
    st = UniversalSimState(len(idF), len(idB), N_R, len(bodies), p.restDensity)
    st.idF[:] = idF; st.xPosF[:] = xF; st.yPosF[:] = yF; st.zPosF[:] = zF
    st.idB[:] = idB; st.xPosB[:] = xB; st.yPosB[:] = yB; st.zPosB[:] = zB
    default_psi = f32(p.massB)
    st.psiB[:] = default_psi
    st.volB[:] = f32(default_psi / f32(p.restDensity))
    if N_R:
        st.xPosRelR[:] = np.concatenate(rel[0]); st.yPosRelR[:] = np.concatenate(rel[1])
        st.zPosRelR[:] = np.concatenate(rel[2]); st.bodyIdR[:] = np.concatenate(body_of)
        st.psiR[:] = default_psi
        st.volR[:] = f32(default_psi / f32(p.restDensity))
        for b, body in enumerate(bodies):
            st.xCM[b], st.yCM[b], st.zCM[b] = body["center"]
            st.massRB[b], st.massInvRB[b] = body["mass"], body["massInv"]
            st.iBodyInv00[b], st.iBodyInv11[b], st.iBodyInv22[b] = body["iBodyInv"]
            A = body["A"]
            for r in range(3):
                for c in range(3):
                    getattr(st, f"a{r}{c}")[b] = A[r, c]
            st.rigidParticleCountRB[b] = int((st.bodyIdR == b).sum())
    dmin, dmax = sim_domain_bounds([container], p)
    return st, dmin, dmax


def dam_scene(n_side, dx, tank, p: SimParams, corner=(0.0, 0.0, 0.0), jitter=0.01, seed=42):
    """Cubic block of n_side^3 lattice particles (spacing dx, +-jitter*dx) in the corner of a
    tank of extent `tank` with 2-layer walls; the block spans n_side*dx per axis."""
    p.jitterFracF = jitter
    p.jitterSeedF = seed
    side = n_side * dx
    container = OBB((0.0, 0.0, 0.0), tuple(tank))
    fluid = OBB(tuple(corner), (side, side, side))
    return breaking_dam(container, fluid, p)


def dam_32k(seed=42):
    """32x32x32 = 32,768 fluid particles, dx = 0.02, 1.6 x 0.8 x 0.8 m tank, dt = 1e-3."""
    from .params import dam_params
    p = dam_params(0.02, 1e-3)
    st, dmin, dmax = dam_scene(32, 0.02, (1.6, 0.8, 0.8), p, seed=seed)
    return st, dmin, dmax, p


def dam_1m(seed=42):
    """100^3 = 1,000,000 fluid particles, dx = 0.01, 5 x 2 x 2 m tank, dt = 5e-4."""
    from .params import dam_params
    p = dam_params(0.01, 5e-4)
    st, dmin, dmax = dam_scene(100, 0.01, (5.0, 2.0, 2.0), p, seed=seed)
    return st, dmin, dmax, p


def uniform_points(n, seed=1):
    rng = np.random.default_rng(seed)
    return rng.random((n, 3), dtype=np.float32)


def clustered_points(n, seed=1, blobs=16, sigma=0.05, background=0.2):
    rng = np.random.default_rng(seed)
    n_bg = int(round(background * n))
    n_bl = n - n_bg
    centres = rng.random((blobs, 3))
    which = rng.integers(0, blobs, n_bl)
    pts = centres[which] + rng.normal(0.0, sigma, (n_bl, 3))
    bg = rng.random((n_bg, 3))
    out = np.concatenate([pts, bg]).astype(np.float32)
    return out[rng.permutation(n)]


def neighbor_search_scene(n, distribution="uniform", seed=1):
    """Neighbor-search-only workload: n fluid points in the unit cube (sim domain = unit
    cube), support radius r = (150 / (4 pi n))^(1/3) for ~50 neighbors, h = r / 2."""
    pts = uniform_points(n, seed) if distribution == "uniform" else clustered_points(n, seed)
    r = (150.0 / (4.0 * math.pi * n)) ** (1.0 / 3.0)
    p = SimParams()
    p.set_particle_size(r / 2.0)
    st = UniversalSimState(n, 0, 0, 0, p.restDensity)
    st.xPosF[:], st.yPosF[:], st.zPosF[:] = pts[:, 0], pts[:, 1], pts[:, 2]
    return st, np.zeros(3, f32), np.ones(3, f32), p


def _rotation(rng):
    """Seeded uniform random rotation (unit quaternion from three uniforms, Shoemake 1992)."""
    u1, u2, u3 = rng.random(3)
    a, b = math.sqrt(1.0 - u1), math.sqrt(u1)
    qw, qx, qy, qz = a * math.sin(2 * math.pi * u2), a * math.cos(2 * math.pi * u2), \
        b * math.sin(2 * math.pi * u3), b * math.cos(2 * math.pi * u3)
    return np.array([
        [1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw)],
        [2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw)],
        [2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)]])


def rigid_dam(block=(100, 125, 80), dx=0.008, tank=(4.0, 1.5, 1.5), cubes=8, edge=0.15, dt=4e-4, seed=7,
              drop_speed=1.0):
    """Two-sided dam with floating hollow cubes: two fluid blocks of block[0] x block[1] x
    block[2] lattice particles (spacing dx) in opposite corners of the tank, `cubes` hollow
    rigid cubes (edge `edge`, 2 particle layers, BuildRigidBody_OBB_Hollow) with seeded random
    orientations resting on the blocks' top faces (half of them on each block, in a 2 x n grid
    over the face, seeded jitter, the lowest rigid particles level with the top fluid layer), dropped
    onto it at `drop_speed` m/s, so fluid-rigid forces act from the first steps; the first half
    of the cubes have density 500 kg/m^3, the rest 2000 kg/m^3. Defaults: 2,000,000 fluid
    particles, 8 cubes of 3,088 particles."""
    from .params import dam_params
    p = dam_params(dx, dt)
    p.jitterFracF = 0.01
    p.jitterSeedF = seed
    ext = [(n + 0.5) * dx for n in block]  # n lattice sites per axis, robust to FP32 rounding
    container = OBB((0.0, 0.0, 0.0), tuple(tank))
    fluids = [OBB((0.0, 0.0, 0.0), tuple(ext)),
              OBB((tank[0] - ext[0], 0.0, tank[2] - ext[2]), tuple(ext))]
    rng = np.random.default_rng(seed)
    per_block = max(1, (cubes + 1) // 2)
    cols = max(1, (per_block + 1) // 2)
    corners = np.array([[i, j, k] for i in (0, 1) for j in (0, 1) for k in (0, 1)], np.float64) * edge
    rigid = []
    for k in range(cubes):
        b, slot = divmod(k, per_block)
        fo = fluids[min(b, 1)].origin
        # cell of a 2 x cols grid over the block's top face, centre jittered by up to a tenth of the cell
        fx = (slot % cols + 0.5 + 0.2 * (rng.random() - 0.5)) / cols
        fz = (slot // cols + 0.5 + 0.2 * (rng.random() - 0.5)) / 2.0
        R = _rotation(rng)
        low = float(((corners - 0.5 * edge) @ R.T)[:, 1].min())  # lowest corner below the centre
        c = np.array([fo[0] + fx * ext[0], ext[1] - 1.25 * dx - low, fo[2] + fz * ext[2]])
        u, v, w = (tuple(float(x) for x in R[:, cc]) for cc in range(3))
        origin = tuple(float(x) for x in c - R @ np.full(3, 0.5 * edge))
        rigid.append((OBB(origin, (edge, edge, edge), u, v, w), 500.0 if k < cubes // 2 else 2000.0))
    st, dmin, dmax = breaking_dam(container, fluids, p, rigid)
    st.yVelRB[:] = -drop_speed
    return st, dmin, dmax, p


def floating_cubes(seed=5, dx=0.03, dt=1e-3):
    """Small rigid-coupling scene: a 30 x 10 x 20 fluid slab (spacing dx) in a 0.9 x 0.6 x 0.6 m
    tank and two hollow cubes (edge 0.18 m, densities 500 and 2000 kg/m^3, seeded random
    orientations) resting on its surface, so fluid-rigid forces act from the first step."""
    from .params import dam_params
    p = dam_params(dx, dt)
    p.jitterFracF = 0.01
    p.jitterSeedF = seed
    container = OBB((0.0, 0.0, 0.0), (0.9, 0.6, 0.6))
    top = (10 + 0.5) * dx
    fluid = OBB((0.0, 0.0, 0.0), ((30 + 0.5) * dx, top, (20 + 0.5) * dx))
    rng = np.random.default_rng(seed)
    rigid = []
    edge = 0.18
    for cx, dens in ((0.25, 500.0), (0.62, 2000.0)):
        R = _rotation(rng)
        c = np.array([cx, top + 0.12, 0.3])
        origin = tuple(float(x) for x in c - R @ np.full(3, 0.5 * edge))
        axes = (tuple(float(x) for x in R[:, j]) for j in range(3))
        rigid.append((OBB(origin, (edge, edge, edge), *axes), dens))
    st, dmin, dmax = breaking_dam(container, fluid, p, rigid)
    return st, dmin, dmax, p


def floating_mesh_body(seed=5, dx=0.03, dt=1e-3, radius=0.1, density=500.0, sampler=None):
    """Mesh rigid-body scene: the floating-cubes fluid slab and tank with one icosphere body
    (radius `radius`, density `density`), sampled from its triangle surface by the mesh surface
    sampler (GPU by default), resting on the fluid surface."""
    from . import mesh as M
    from .params import dam_params
    p = dam_params(dx, dt)
    p.jitterFracF = 0.01
    p.jitterSeedF = seed
    container = OBB((0.0, 0.0, 0.0), (0.9, 0.6, 0.6))
    top = (10 + 0.5) * dx
    fluid = OBB((0.0, 0.0, 0.0), ((30 + 0.5) * dx, top, (20 + 0.5) * dx))
    st, dmin, dmax = breaking_dam(container, fluid, p)
    st, _ = M.build_rigid_mesh(st, M.icosphere(1.0, 2), p, 2.0 * radius, density, (0.45, top + radius + 0.6 * dx, 0.3),
                               M.euler_orientation(20.0, 10.0, 5.0), sampler=sampler)
    return st, dmin, dmax, p


@dataclasses.dataclass
class ServedSceneSpec:
    """One scene of the served stream: a block of nx x ny x nz fluid particles (spacing dx)
    in the corner of a tank twice the block's extent per axis, arriving at `arrival_s`."""
    index: int
    nx: int
    ny: int
    nz: int
    dx: float
    dt: float
    arrival_s: float
    seed: int

    @property
    def n_fluid(self) -> int:
        return self.nx * self.ny * self.nz

    def build(self):
        from .params import dam_params
        p = dam_params(self.dx, self.dt)
        p.jitterFracF = 0.01
        p.jitterSeedF = self.seed
        ext = [(n + 0.5) * self.dx for n in (self.nx, self.ny, self.nz)]
        container = OBB((0.0, 0.0, 0.0), tuple(2.0 * e for e in ext))
        st, dmin, dmax = breaking_dam(container, OBB((0.0, 0.0, 0.0), tuple(ext)), p)
        return st, dmin, dmax, p


def served_stream(n_scenes=256, n_min=4096, n_max=262144, dx=0.01, dt=5e-4, rate_hz=64.0, seed=2024):
    """Seeded served-stream workload: N_F log-uniform in [n_min, n_max], block aspect ratios
    nx/ny and nz/ny uniform in [0.5, 2], Poisson arrivals at `rate_hz` scenes per second."""
    rng = np.random.default_rng(seed)
    specs, t = [], 0.0
    for k in range(n_scenes):
        n = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
        r1, r2 = rng.uniform(0.5, 2.0, 2)
        ny = max(2, int(round((n / (r1 * r2)) ** (1.0 / 3.0))))
        nx = max(2, int(round(r1 * ny)))
        nz = max(2, int(round(r2 * ny)))
        t += rng.exponential(1.0 / rate_hz) if rate_hz > 0 else 0.0
        specs.append(ServedSceneSpec(k, nx, ny, nz, dx, dt, t, seed * 1000 + k))
    return specs


def stacked_cubes(dx=0.02, dt=1e-3, edge=0.16, seed=9, tilt_deg=6.0, overlap=0.008, drop_speed=0.5):
    """Rigid-contact scene: a hollow cube pressed `overlap` into the tank floor and a second,
    slightly tilted one pressed into it and moving down at `drop_speed` (2 particle layers each,
    densities 1000 and 700 kg/m^3), in a 0.6 m tank with a small fluid block in a far corner.
    The contact density exceeds 1 from the first step, so the rigid contact solver
    (rigid_solver.cpp:602) iterates every step."""
    from .params import dam_params
    p = dam_params(dx, dt)
    p.jitterFracF = 0.01
    p.jitterSeedF = seed
    container = OBB((0.0, 0.0, 0.0), (0.6, 0.6, 0.6))
    fluid = OBB((0.0, 0.0, 0.0), (6.5 * dx, 4.5 * dx, 6.5 * dx))
    half = 0.5 * edge
    t = math.radians(tilt_deg)
    R = np.array([[math.cos(t), -math.sin(t), 0.0], [math.sin(t), math.cos(t), 0.0], [0.0, 0.0, 1.0]])
    rigid = []
    for c, Rm, dens in ((np.array([0.36, half - overlap, 0.36]), np.eye(3), 1000.0),
                        (np.array([0.37, edge + half - 2.0 * overlap, 0.36]), R, 700.0)):
        origin = tuple(float(x) for x in c - Rm @ np.full(3, half))
        axes = (tuple(float(x) for x in Rm[:, j]) for j in range(3))
        rigid.append((OBB(origin, (edge, edge, edge), *axes), dens))
    st, dmin, dmax = breaking_dam(container, fluid, p, rigid)
    st.yVelRB[1] = -float(drop_speed)
    st.yAngMomRB[:] = 0.0
    return st, dmin, dmax, p
