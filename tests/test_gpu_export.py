"""Export snapshot packing on the GPU (tsp_b200_pack_export_snapshot).

- Bit-exact against a numpy restatement over the GPU's own state and neighbor rows: the set and
  order of exported fluid particles, their positions, and |v| (FP32 products and sums rounded
  separately, then sqrt -- numpy's float32 arithmetic is the same IEEE rounding).
- Against the oracle after the same steps: identical exported count and mesh flags (the
  neighbor counts are bit-exact), positions / velocity magnitudes within the step tolerance
  (FP32 neighbor sums in a different order: 1e-5 m, 1e-4 m/s).
- Rigid particles (floating cubes): world positions, volumes and body indices of every rigid
  particle, compared with the pushed state.
"""
import numpy as np
import pytest

from oracle import OracleBackend
from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.backend import SimBackendB200

pytestmark = pytest.mark.gpu


def loaded(builder, threshold=27, oracle=False):
    st, dmin, dmax, p = builder()
    p = p.copy(surfaceNbrCountThreshold=threshold)
    bes = [SimBackendB200(p)] + ([OracleBackend(p)] if oracle else [])
    for be in bes:
        be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)
        be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    return bes, p, st


def expected_surface(be, threshold):
    rows = [be.rows(k) for k in (abi.LIST_FF, abi.LIST_FB, abi.LIST_FR)]
    cnt = [np.diff(off.astype(np.int64)) for off, _ in rows]
    near = (cnt[1] > 0) | (cnt[2] > 0) | (cnt[0] < threshold)
    flag = near.copy()
    off, idx = rows[0][0].astype(np.int64), rows[0][1]
    for i in np.nonzero(near)[0]:
        flag[idx[off[i]:off[i + 1]]] = True
    return flag


def test_gpu_export_before_first_step_has_no_fluid():
    (g,), p, st = loaded(S.dam_32k)
    snap = g.pack_export_snapshot(p)
    assert snap.N_F == 0 and snap.N_B == st.N_B


@pytest.mark.parametrize("threshold", [20, 27])
def test_gpu_export_bit_exact_against_own_state(threshold):
    (g,), p, st = loaded(S.dam_32k, threshold)
    for _ in range(4):
        g.step(p)
    s = g.push()
    flag = expected_surface(g, threshold)
    mesh_begin = int(st.idB.min()) + 500
    snap = g.pack_export_snapshot(p, include_b=True, mesh_id_begin_b=mesh_begin)
    assert (snap.simStep, snap.simTime) == (s.step, s.time)
    assert 0 < snap.N_F == int(flag.sum()) < st.N_F
    for c in ("xPosF", "yPosF", "zPosF"):
        np.testing.assert_array_equal(getattr(snap, c), getattr(s, c)[flag], c)
    vx, vy, vz = s.xVelF[flag], s.yVelF[flag], s.zVelF[flag]
    np.testing.assert_array_equal(snap.velMagF, np.sqrt(vx * vx + vy * vy + vz * vz))
    assert snap.N_B == st.N_B
    np.testing.assert_array_equal(snap.xPosB, s.xPosB)
    np.testing.assert_array_equal(snap.volB, s.volB)
    np.testing.assert_array_equal(snap.isMeshB, (s.idB >= mesh_begin).astype(np.uint8))
    assert g.pack_export_snapshot(p, include_b=False).N_B == 0


def test_gpu_export_matches_oracle():
    (g, o), p, st = loaded(S.dam_32k, oracle=True)
    for _ in range(3):
        g.step(p)
        o.step(p)
    a, b = g.pack_export_snapshot(p), o.pack_export_snapshot(p)
    assert a.N_F == b.N_F > 0
    for c in ("xPosF", "yPosF", "zPosF"):
        assert np.max(np.abs(getattr(a, c) - getattr(b, c))) <= 1e-5, c
    assert np.max(np.abs(a.velMagF - b.velMagF)) <= 1e-4
    np.testing.assert_array_equal(a.isMeshB, b.isMeshB)


def test_gpu_export_rigid_particles():
    (g,), p, st = loaded(S.floating_cubes)
    for _ in range(3):
        g.step(p)
    s = g.push()
    snap = g.pack_export_snapshot(p)
    assert snap.N_R == st.N_R > 0
    for c in ("xPosR", "yPosR", "zPosR", "volR"):
        np.testing.assert_array_equal(getattr(snap, c), getattr(s, c), c)
    np.testing.assert_array_equal(snap.bodyIdR, s.bodyIdR)
