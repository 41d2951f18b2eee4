"""Export snapshot files in the reference's TSPSNP4 layout and their XDMF views, so particle
output of this backend (one scene or a served batch scene) opens in the same readers.

Layout (source/eval/serial/snapshot_format.h; serialization.cpp:301-360, 1232-1400): a packed
64-byte little-endian header `BinHeaderSnap` {magic "TSPSNP4\\0", endian tag 0x01020304, header
bytes 64, step u64, time f64, N_F, N_B, N_R, N_rankF u64}, then
- particle_data_step_<step, 9 digits>.bin: posF (XYZ triples, f32), velMagF (f32), rankF (u16,
  only in distributed runs), posR (XYZ triples), volR (f32), bodyIdR (u32); N_B is informational;
- static_boundary.bin (boundary particles never move, one file per run): posB (XYZ), volB (f32),
  isMeshB (u8), with N_F = N_R = N_rankF = 0;
- fluid_surface.xdmf / rigid_particles.xdmf: temporal collections over every valid snapshot of
  the directory, ordered by (time, step); static_boundary.xdmf: one grid without a time.
"""
from __future__ import annotations

import os
import struct

import numpy as np

from .state import ExportSnapshot

MAGIC = b"TSPSNP4\x00"
ENDIAN_TAG = 0x01020304
HEADER = struct.Struct("<8sIIQdQQQQ")
assert HEADER.size == 64
U64_MAX = (1 << 64) - 1
MAX_LOCAL_PARTICLE_COUNT = (1 << 31) - 1
STATIC_BOUNDARY_BIN = "static_boundary.bin"
SNAPSHOT_PREFIX, SNAPSHOT_SUFFIX = "particle_data_step_", ".bin"


class ExportFormatError(RuntimeError):
    """A snapshot layout the reference's writer or reader rejects."""


def _append(at, count, width, context):
    if count < 0 or count > U64_MAX or count * width > U64_MAX:
        raise ExportFormatError(f"{context} byte size overflow.")
    if at + count * width > U64_MAX:
        raise ExportFormatError(f"{context} offsets byte size overflow.")
    return at, at + count * width


def compute_export_snapshot_offsets(N_F=0, N_B=0, N_R=0, N_rankF=0) -> dict:
    """ComputeExportSnapshotOffsets (serialization.cpp:301-326); an absent rank array takes no
    space, so the rigid arrays follow the fluid arrays directly."""
    off, at = {}, HEADER.size
    for name, n, w in (("posF", N_F, 12), ("vF", N_F, 4), ("rankF", N_rankF, 2), ("posR", N_R, 12),
                       ("volR", N_R, 4), ("bodyIdR", N_R, 4)):
        off[name], at = _append(at, n, w, "snapshot field")
    off["totalBytes"] = at
    return off


def compute_static_boundary_offsets(N_B=0) -> dict:
    """ComputeStaticBoundaryOffsets (serialization.cpp:328-349)."""
    off, at = {}, HEADER.size
    for name, n, w in (("posB", N_B, 12), ("volB", N_B, 4), ("isMeshB", N_B, 1)):
        off[name], at = _append(at, n, w, "static boundary field")
    off["totalBytes"] = at
    return off


def compute_distributed_export_layout(rank_counts, rank: int) -> dict:
    """ComputeDistributedExportLayout (serialization.cpp:370-402): per population (F, B, R)
    the global total, this rank's first index and the largest local count."""
    n_ranks = len(rank_counts) // 3
    if len(rank_counts) % 3 or n_ranks == 0 or n_ranks > 1 + 0xFFFF or rank < 0 or rank >= n_ranks:
        raise ExportFormatError("Invalid distributed snapshot count table.")
    total, begin, mx = [0, 0, 0], [0, 0, 0], [0, 0, 0]
    for r in range(n_ranks):
        for p in range(3):
            n = int(rank_counts[3 * r + p])
            if n > MAX_LOCAL_PARTICLE_COUNT:
                raise OverflowError("rank-local export count exceeds the local particle limit.")
            if r == rank:
                begin[p] = total[p]
            total[p] += n
            mx[p] = max(mx[p], n)
    return {"N_total": total, "beginIdx": begin, "N_max": mx}


def snapshot_file_name(step: int) -> str:
    return f"{SNAPSHOT_PREFIX}{int(step):09d}{SNAPSHOT_SUFFIX}"


def _header(step, time, n_f, n_b, n_r, n_rank):
    return HEADER.pack(MAGIC, ENDIAN_TAG, HEADER.size, int(step), float(time), n_f, n_b, n_r, n_rank)


def _xyz(x, y, z):
    return np.stack([np.asarray(x, "<f4"), np.asarray(y, "<f4"), np.asarray(z, "<f4")], axis=1).tobytes()


def _write_atomic(path, chunks, atomic=True, temp_suffix=".tmp"):
    tmp = path + temp_suffix if atomic else path
    try:
        with open(tmp, "wb") as f:
            for c in chunks:
                f.write(c)
    except BaseException:
        if atomic and os.path.exists(tmp):
            os.remove(tmp)
        raise
    if atomic:
        os.replace(tmp, path)


def save_boundary_bin(snap: ExportSnapshot, directory: str, atomic=True):
    """SaveBoundaryBin (serialization.cpp:1232-1284): a run without boundary particles removes
    the file."""
    if snap.isMeshB.size != snap.N_B:
        raise ExportFormatError("Inconsistent boundary classification count.")
    path = os.path.join(directory, STATIC_BOUNDARY_BIN)
    if snap.N_B == 0:
        if os.path.exists(path):
            os.remove(path)
        return
    _write_atomic(path, [_header(snap.simStep, snap.simTime, 0, snap.N_B, 0, 0),
                         _xyz(snap.xPosB, snap.yPosB, snap.zPosB), np.asarray(snap.volB, "<f4").tobytes(),
                         np.asarray(snap.isMeshB, np.uint8).tobytes()], atomic)


def save_export_snapshot(snap: ExportSnapshot, directory: str, include_b: bool = True, atomic=True) -> str:
    """SaveExportSnapshot (serialization.cpp:1286-1400): returns the path of the snapshot file."""
    os.makedirs(directory, exist_ok=True)
    for name, n in (("xPosF", snap.N_F), ("yPosF", snap.N_F), ("zPosF", snap.N_F), ("velMagF", snap.N_F),
                    ("xPosR", snap.N_R), ("yPosR", snap.N_R), ("zPosR", snap.N_R), ("volR", snap.N_R),
                    ("bodyIdR", snap.N_R)):
        if np.asarray(getattr(snap, name)).size != n:
            raise ExportFormatError(f"Snapshot array '{name}' does not match its count {n}.")
    n_rank = int(snap.rankF.size)
    if n_rank not in (0, snap.N_F):
        raise ExportFormatError("Snapshot rank array does not match the fluid count.")
    if include_b:
        save_boundary_bin(snap, directory, atomic)
    path = os.path.join(directory, snapshot_file_name(snap.simStep))
    _write_atomic(path, [_header(snap.simStep, snap.simTime, snap.N_F, snap.N_B, snap.N_R, n_rank),
                         _xyz(snap.xPosF, snap.yPosF, snap.zPosF), np.asarray(snap.velMagF, "<f4").tobytes(),
                         np.asarray(snap.rankF, "<u2").tobytes(), _xyz(snap.xPosR, snap.yPosR, snap.zPosR),
                         np.asarray(snap.volR, "<f4").tobytes(), np.asarray(snap.bodyIdR, "<u4").tobytes()], atomic)
    return path


def read_snapshot_info(path: str, boundary: bool = False):
    """TryReadExportSnapshotBinInfo / TryReadStaticBoundaryBinInfo (serialization.cpp:415-490):
    header fields of a valid file, or None for a file of another layout or a truncated one."""
    try:
        size = os.path.getsize(path)
        with open(path, "rb") as f:
            raw = f.read(HEADER.size)
    except OSError:
        return None
    if len(raw) != HEADER.size:
        return None
    magic, tag, hb, step, time, n_f, n_b, n_r, n_rank = HEADER.unpack(raw)
    if magic != MAGIC or tag != ENDIAN_TAG or hb != HEADER.size:
        return None
    info = {"fileName": os.path.basename(path), "step": step, "time": time, "N_F": n_f, "N_B": n_b, "N_R": n_r,
            "N_rankF": n_rank}
    try:
        if boundary:
            if n_f or n_r or n_rank:
                return None
            total = compute_static_boundary_offsets(n_b)["totalBytes"]
        else:
            if n_rank not in (0, n_f):
                return None
            total = compute_export_snapshot_offsets(n_f, n_b, n_r, n_rank)["totalBytes"]
    except ExportFormatError:
        return None
    return info if size == total else None


def load_export_snapshot(path: str, boundary_path: str | None = None) -> ExportSnapshot:
    """Read a snapshot file (and optionally the static boundary file) back into an ExportSnapshot."""
    info = read_snapshot_info(path)
    if info is None:
        raise ExportFormatError(f"Invalid export snapshot '{path}'.")
    off = compute_export_snapshot_offsets(info["N_F"], info["N_B"], info["N_R"], info["N_rankF"])
    data = open(path, "rb").read()
    snap = ExportSnapshot(info["N_F"], 0, info["N_R"])
    snap.simStep, snap.simTime = info["step"], info["time"]
    xyz = np.frombuffer(data, "<f4", 3 * info["N_F"], off["posF"]).reshape(-1, 3)
    snap.xPosF, snap.yPosF, snap.zPosF = (xyz[:, k].copy() for k in range(3))
    snap.velMagF = np.frombuffer(data, "<f4", info["N_F"], off["vF"]).copy()
    snap.rankF = np.frombuffer(data, "<u2", info["N_rankF"], off["rankF"]).copy()
    xyz = np.frombuffer(data, "<f4", 3 * info["N_R"], off["posR"]).reshape(-1, 3)
    snap.xPosR, snap.yPosR, snap.zPosR = (xyz[:, k].copy() for k in range(3))
    snap.volR = np.frombuffer(data, "<f4", info["N_R"], off["volR"]).copy()
    snap.bodyIdR = np.frombuffer(data, "<u4", info["N_R"], off["bodyIdR"]).copy()
    if boundary_path is not None:
        binfo = read_snapshot_info(boundary_path, boundary=True)
        if binfo is None:
            raise ExportFormatError(f"Invalid static boundary file '{boundary_path}'.")
        boff = compute_static_boundary_offsets(binfo["N_B"])
        bdata = open(boundary_path, "rb").read()
        n = binfo["N_B"]
        xyz = np.frombuffer(bdata, "<f4", 3 * n, boff["posB"]).reshape(-1, 3)
        snap.xPosB, snap.yPosB, snap.zPosB = (xyz[:, k].copy() for k in range(3))
        snap.volB = np.frombuffer(bdata, "<f4", n, boff["volB"]).copy()
        snap.isMeshB = np.frombuffer(bdata, np.uint8, n, boff["isMeshB"]).copy()
        snap.N_B = n
    return snap


def collect_snapshot_infos(directory: str):
    """CollectExportSnapshotBinInfos (serialization.cpp:492-548): every valid snapshot of the
    directory, ordered by (time, step); files of another layout are skipped."""
    infos = []
    for name in os.listdir(directory):
        if not (name.startswith(SNAPSHOT_PREFIX) and name.endswith(SNAPSHOT_SUFFIX)):
            continue
        full = os.path.join(directory, name)
        if not os.path.isfile(full):
            continue
        info = read_snapshot_info(full)
        if info is not None:
            infos.append(info)
    infos.sort(key=lambda i: (i["time"], i["step"]))
    return infos


def _data_item(dims, number_type, precision, offset, file_name, indent):
    return (f'{indent}<DataItem Dimensions="{dims}" NumberType="{number_type}" Precision="{precision}" '
            f'Format="Binary" Endian="Little" Seek="{offset}">\n{indent}  {file_name}\n{indent}</DataItem>\n')


def _geometry(name, n, offset, file_name):
    return (f'        <Geometry Name="{name}" GeometryType="XYZ">\n'
            + _data_item(f"{n} 3", "Float", 4, offset, file_name, "          ") + "        </Geometry>\n")


def _attribute(name, n, number_type, precision, offset, file_name):
    return (f'        <Attribute Name="{name}" AttributeType="Scalar" Center="Node">\n'
            + _data_item(str(n), number_type, precision, offset, file_name, "          ")
            + "        </Attribute>\n")


def _time(t):
    return f'        <Time Value="{float(t):.16g}" />\n'


def _fluid_grid(i):
    off = compute_export_snapshot_offsets(i["N_F"], i["N_B"], i["N_R"], i["N_rankF"])
    s = '      <Grid Name="FluidSurface" GridType="Uniform">\n' + _time(i["time"])
    s += f'        <Topology TopologyType="Polyvertex" Dimensions="{i["N_F"]}"/>\n'
    s += _geometry("posF", i["N_F"], off["posF"], i["fileName"])
    s += _attribute("velMagF", i["N_F"], "Float", 4, off["vF"], i["fileName"])
    if i["N_rankF"] > 0:
        s += _attribute("rankF", i["N_F"], "UShort", 2, off["rankF"], i["fileName"])
    return s + "      </Grid>\n"


def _rigid_grid(i):
    off = compute_export_snapshot_offsets(i["N_F"], i["N_B"], i["N_R"], i["N_rankF"])
    s = '      <Grid Name="RigidParticles" GridType="Uniform">\n' + _time(i["time"])
    s += f'        <Topology TopologyType="Polyvertex" Dimensions="{i["N_R"]}"/>\n'
    s += _geometry("posR", i["N_R"], off["posR"], i["fileName"])
    s += _attribute("volR", i["N_R"], "Float", 4, off["volR"], i["fileName"])
    s += _attribute("bodyIdR", i["N_R"], "UInt", 4, off["bodyIdR"], i["fileName"])
    return s + "      </Grid>\n"


def _boundary_grid(i):
    off = compute_static_boundary_offsets(i["N_B"])
    s = '      <Grid Name="StaticBoundary" GridType="Uniform">\n'
    s += f'        <Topology TopologyType="Polyvertex" Dimensions="{i["N_B"]}"/>\n'
    s += _geometry("posB", i["N_B"], off["posB"], STATIC_BOUNDARY_BIN)
    s += _attribute("volB", i["N_B"], "Float", 4, off["volB"], STATIC_BOUNDARY_BIN)
    s += _attribute("isMeshB", i["N_B"], "UChar", 1, off["isMeshB"], STATIC_BOUNDARY_BIN)
    return s + "      </Grid>\n"


def _xdmf(body):
    return '<?xml version="1.0" ?>\n<Xdmf Version="3.0">\n  <Domain>\n' + body + "  </Domain>\n</Xdmf>\n"


def _collection(name, infos, grid):
    return (f'    <Grid Name="{name}" GridType="Collection" CollectionType="Temporal">\n'
            + "".join(grid(i) for i in infos) + "    </Grid>\n")


def save_export_snapshot_xdmf_views(directory: str, atomic=True):
    """SaveExportSnapshotXdmfViews (serialization.cpp:1554-1645): rebuild fluid_surface.xdmf,
    static_boundary.xdmf (when a valid boundary file exists) and rigid_particles.xdmf (when any
    snapshot holds rigid particles) from the snapshot files of `directory`."""
    infos = collect_snapshot_infos(directory)
    if not infos:
        raise ExportFormatError(f"No export snapshot binary files found in '{directory}'.")
    _write_atomic(os.path.join(directory, "fluid_surface.xdmf"),
                  [_xdmf(_collection("FluidSurface", infos, _fluid_grid)).encode()], atomic)
    binfo = read_snapshot_info(os.path.join(directory, STATIC_BOUNDARY_BIN), boundary=True)
    bpath = os.path.join(directory, "static_boundary.xdmf")
    if binfo is not None:
        _write_atomic(bpath, [_xdmf(_boundary_grid(binfo)).encode()], atomic)
    elif os.path.exists(bpath):
        os.remove(bpath)
    rpath = os.path.join(directory, "rigid_particles.xdmf")
    if any(i["N_R"] > 0 for i in infos):
        _write_atomic(rpath, [_xdmf(_collection("RigidParticles", infos, _rigid_grid)).encode()], atomic)
    elif os.path.exists(rpath):
        os.remove(rpath)
