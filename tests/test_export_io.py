"""Export snapshot files (TSPSNP4) and XDMF views: the reference's layout known answers
(tests/unit/snapshot_format.cpp) and the oracle's surface classification against an
independent restatement over its own neighbor rows."""
import os
import struct

import numpy as np
import pytest

from oracle import OracleBackend
from turbospharticles_b200 import abi, scene as S
from turbospharticles_b200.export_io import (ExportFormatError, collect_snapshot_infos,
                                             compute_distributed_export_layout, compute_export_snapshot_offsets,
                                             compute_static_boundary_offsets, load_export_snapshot,
                                             read_snapshot_info, save_export_snapshot,
                                             save_export_snapshot_xdmf_views, snapshot_file_name)
from turbospharticles_b200.state import ExportSnapshot

U64_MAX = (1 << 64) - 1


def test_empty_populations_contain_only_header():
    o, b = compute_export_snapshot_offsets(), compute_static_boundary_offsets()
    assert set(o.values()) == {64} and set(b.values()) == {64}


def test_computes_mixed_population_offsets():
    o = compute_export_snapshot_offsets(N_F=2, N_rankF=2, N_R=3)
    assert [o[k] for k in ("posF", "vF", "rankF", "posR", "volR", "bodyIdR", "totalBytes")] == \
        [64, 88, 96, 100, 136, 148, 160]


def test_omits_absent_rank_storage():
    o = compute_export_snapshot_offsets(N_F=2, N_R=3)
    assert [o[k] for k in ("posR", "volR", "bodyIdR", "totalBytes")] == [96, 132, 144, 156]


def test_computes_static_boundary_offsets():
    b = compute_static_boundary_offsets(5)
    assert [b[k] for k in ("posB", "volB", "isMeshB", "totalBytes")] == [64, 124, 144, 149]


def test_keeps_offsets_wider_than_32_bits():
    o = compute_export_snapshot_offsets(N_F=268_435_456)
    assert (o["vF"], o["posR"], o["totalBytes"]) == (3_221_225_536, 4_294_967_360, 4_294_967_360)


def test_rejects_field_size_overflow():
    with pytest.raises(ExportFormatError):
        compute_export_snapshot_offsets(N_F=U64_MAX, N_B=U64_MAX)
    with pytest.raises(ExportFormatError):
        compute_static_boundary_offsets(U64_MAX)


def test_rejects_combined_size_overflow():
    with pytest.raises(ExportFormatError):
        compute_export_snapshot_offsets(N_F=U64_MAX // 16)


@pytest.mark.parametrize("rank,begin", [(0, [0, 0, 0]), (1, [2, 1, 0]), (2, [2, 4, 1])])
def test_computes_distributed_population_layout(rank, begin):
    lay = compute_distributed_export_layout([2, 1, 0, 0, 3, 1, 4, 0, 2], rank)
    assert lay["N_total"] == [6, 4, 3] and lay["N_max"] == [4, 3, 2] and lay["beginIdx"] == begin


@pytest.mark.parametrize("counts,rank", [([], 0), ([1, 2], 0), ([1, 2, 3], -1), ([1, 2, 3], 1)])
def test_rejects_malformed_distributed_tables(counts, rank):
    with pytest.raises(ExportFormatError):
        compute_distributed_export_layout(counts, rank)


def test_distributed_rank_id_range():
    compute_distributed_export_layout([0] * (3 * 65_536), 65_535)
    with pytest.raises(ExportFormatError):
        compute_distributed_export_layout([0] * (3 * 65_537), 0)
    with pytest.raises(OverflowError):
        compute_distributed_export_layout([2_147_483_648, 0, 0], 0)


def mixed_snapshot(n_f=2, n_b=5, n_r=3, step=1234, time=0.0625):
    s = ExportSnapshot(n_f, n_b, n_r)
    s.simStep, s.simTime = step, time
    for k, name in enumerate(("xPosF", "yPosF", "zPosF", "velMagF", "xPosB", "yPosB", "zPosB", "volB",
                              "xPosR", "yPosR", "zPosR", "volR")):
        a = getattr(s, name)
        a[:] = 10.0 * k + np.arange(a.size, dtype=np.float32) + np.float32(0.5)
    s.isMeshB[:] = [0, 1, 0, 1, 1][:n_b]
    s.bodyIdR[:] = np.arange(n_r) % 2
    return s


def test_snapshot_files_have_the_documented_bytes(tmp_path):
    s = mixed_snapshot()
    path = save_export_snapshot(s, str(tmp_path))
    assert os.path.basename(path) == "particle_data_step_000001234.bin" == snapshot_file_name(1234)
    exp = b"TSPSNP4\x00" + struct.pack("<IIQdQQQQ", 0x01020304, 64, 1234, 0.0625, 2, 5, 3, 0)
    for i in range(2):
        exp += struct.pack("<3f", s.xPosF[i], s.yPosF[i], s.zPosF[i])
    exp += s.velMagF.astype("<f4").tobytes()
    for i in range(3):
        exp += struct.pack("<3f", s.xPosR[i], s.yPosR[i], s.zPosR[i])
    exp += s.volR.astype("<f4").tobytes() + s.bodyIdR.astype("<u4").tobytes()
    assert len(exp) == 156
    assert open(path, "rb").read() == exp
    bexp = b"TSPSNP4\x00" + struct.pack("<IIQdQQQQ", 0x01020304, 64, 1234, 0.0625, 0, 5, 0, 0)
    for i in range(5):
        bexp += struct.pack("<3f", s.xPosB[i], s.yPosB[i], s.zPosB[i])
    bexp += s.volB.astype("<f4").tobytes() + s.isMeshB.tobytes()
    assert len(bexp) == 149
    assert (tmp_path / "static_boundary.bin").read_bytes() == bexp


def test_snapshot_round_trip_and_boundary_removal(tmp_path):
    s = mixed_snapshot()
    path = save_export_snapshot(s, str(tmp_path))
    r = load_export_snapshot(path, str(tmp_path / "static_boundary.bin"))
    for n in ("xPosF", "yPosF", "zPosF", "velMagF", "xPosB", "yPosB", "zPosB", "volB", "isMeshB", "xPosR",
              "yPosR", "zPosR", "volR", "bodyIdR"):
        np.testing.assert_array_equal(getattr(r, n), getattr(s, n), n)
    assert (r.simStep, r.simTime, r.N_F, r.N_B, r.N_R) == (1234, 0.0625, 2, 5, 3)
    save_export_snapshot(mixed_snapshot(n_b=0, step=1235), str(tmp_path))
    assert not (tmp_path / "static_boundary.bin").exists()


def test_xdmf_views_reference_every_valid_snapshot(tmp_path):
    d = str(tmp_path)
    save_export_snapshot(mixed_snapshot(step=20, time=0.02), d)
    save_export_snapshot(mixed_snapshot(n_f=4, step=10, time=0.01), d)
    (tmp_path / "particle_data_step_000000030.bin").write_bytes(b"not a snapshot")  # skipped
    assert [i["step"] for i in collect_snapshot_infos(d)] == [10, 20]
    save_export_snapshot_xdmf_views(d)
    fluid = (tmp_path / "fluid_surface.xdmf").read_text()
    assert fluid.startswith('<?xml version="1.0" ?>\n<Xdmf Version="3.0">\n  <Domain>\n')
    assert fluid.count('<Grid Name="FluidSurface" GridType="Uniform">') == 2
    assert fluid.index("particle_data_step_000000010.bin") < fluid.index("particle_data_step_000000020.bin")
    assert '<Time Value="0.01" />' in fluid and 'Dimensions="4 3"' in fluid
    assert 'Name="velMagF"' in fluid and 'Seek="112"' in fluid  # 64 + 4 * 12 for the 4-particle file
    rigid = (tmp_path / "rigid_particles.xdmf").read_text()
    assert 'Name="bodyIdR"' in rigid and 'NumberType="UInt"' in rigid
    bnd = (tmp_path / "static_boundary.xdmf").read_text()
    assert '<Time' not in bnd and 'Name="isMeshB"' in bnd and 'NumberType="UChar"' in bnd
    assert read_snapshot_info(str(tmp_path / "static_boundary.bin"), boundary=True)["N_B"] == 5


def surface_restated(counts_ff, counts_fb, counts_fr, off_ff, idx_ff, threshold):
    """IsNearSurfaceFluidParticle + ClassifyExportSurfaceParticles over CSR rows."""
    near = (counts_fb > 0) | (counts_fr > 0) | (counts_ff < threshold)
    flag = near.copy()
    for i in np.nonzero(near)[0]:
        flag[idx_ff[off_ff[i]:off_ff[i + 1]]] = True
    return flag


@pytest.mark.parametrize("threshold", [20, 27, 33])
def test_oracle_export_classification_matches_restatement(threshold):
    st, dmin, dmax, p = S.dam_32k()
    p = p.copy(surfaceNbrCountThreshold=threshold)
    o = OracleBackend(p)
    o.set_sim_domain_bounds(dmin, dmax)
    o.pull(st, p)
    o.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    o.step(p)
    rows = [o.rows(k) for k in (abi.LIST_FF, abi.LIST_FB, abi.LIST_FR)]
    cnt = [np.diff(off.astype(np.int64)) for off, _ in rows]
    flag = surface_restated(cnt[0], cnt[1], cnt[2], rows[0][0].astype(np.int64), rows[0][1], threshold)
    snap = o.pack_export_snapshot(p, include_b=True, mesh_id_begin_b=int(st.idB.min()) + 100)
    s = o.push()
    assert 0 < snap.N_F == int(flag.sum()) <= st.N_F
    np.testing.assert_array_equal(snap.xPosF, s.xPosF[flag])
    vx, vy, vz = s.xVelF[flag], s.yVelF[flag], s.zVelF[flag]
    np.testing.assert_array_equal(snap.velMagF, np.sqrt(vx * vx + vy * vy + vz * vz))
    assert snap.N_B == st.N_B and snap.N_R == 0
    np.testing.assert_array_equal(snap.isMeshB, (s.idB >= int(st.idB.min()) + 100).astype(np.uint8))
    assert o.pack_export_snapshot(p, include_b=False).N_B == 0
