"""Simulation-state files in the reference's TSPSIM2 format, so scenes run on this backend
(one-scene or served batch) can be saved, resumed and exchanged with the reference.

Format (source/eval/serial/state_format.h, serialization.cpp:160-235, 838-935): a packed
64-byte little-endian header `BinHeaderSim` {magic "TSPSIM2\\0", endian tag 0x01020304, header
bytes 64, step u64, time f64, N_F, N_B, N_R, N_RB u64}, then each population's arrays one after
the other in a fixed field order: fluid {id u64, 16 x f32}, boundary {id u64, 5 x f32}, rigid
particles {id u64, bodyId u32, 5 x f32}, rigid bodies {id u32, rigidParticleCount u32,
32 x f32} -- 72, 28, 32 and 136 bytes per element. Loading checks the header, the step/time,
the exact file length, that no particle carries the invalid ID 2^64 - 1 and that the rigid
attachments are consistent, like the reference's loader; saving checks the same state rules.
The rigid particles' world positions (xPosR/yPosR/zPosR) are not part of the format: they
follow from the body transform and are zero after a load, as in the reference's state.
"""
from __future__ import annotations

import math
import os
import struct

import numpy as np

from .state import BODY_F32, BOUNDARY_F32, FLUID_F32, UniversalSimState

MAGIC = b"TSPSIM2\x00"
ENDIAN_TAG = 0x01020304
HEADER = struct.Struct("<8sIIQdQQQQ")
assert HEADER.size == 64
INVALID_PARTICLE_ID = np.uint64(0xFFFFFFFFFFFFFFFF)
U64_MAX = (1 << 64) - 1
U32_MAX = (1 << 32) - 1
MAX_LOCAL_PARTICLE_COUNT = (1 << 31) - 1  # Sim::MaxLocalParticleCount (particle_types.h:17)

# bytes per element of each population (ComputeSimStateOffsets, serialization.cpp:193-211)
BYTES_F = 8 + 16 * 4
BYTES_B = 8 + 5 * 4
BYTES_R = 8 + 4 + 5 * 4
BYTES_RB = 2 * 4 + 32 * 4
RIGID_FIELDS = ["xPosRelR", "yPosRelR", "zPosRelR", "volR", "psiR"]


class SimStateError(RuntimeError):
    """A state file or state that the reference's loader / writer would reject."""


def compute_sim_state_offsets(n_f: int, n_b: int, n_r: int, n_rb: int) -> dict:
    """Byte offsets of the four populations and the total length; overflow of u64 is an error
    (CheckedByteProduct / CheckedByteSum)."""
    off, at = {}, HEADER.size
    for name, n, per in (("fluid", n_f, BYTES_F), ("boundary", n_b, BYTES_B), ("rigid", n_r, BYTES_R),
                         ("rigidBodies", n_rb, BYTES_RB)):
        if n < 0 or n > U64_MAX:
            raise SimStateError(f"{name} count out of range")
        size = n * per
        if size > U64_MAX or at + size > U64_MAX:
            raise SimStateError("simulation state size overflows 64 bits")
        off[name] = at
        at += size
    off["totalBytes"] = at
    return off


def make_header(step: int, time: float, n_f: int, n_b: int, n_r: int, n_rb: int) -> bytes:
    return HEADER.pack(MAGIC, ENDIAN_TAG, HEADER.size, step, time, n_f, n_b, n_r, n_rb)


def _validate_ids(st: UniversalSimState):
    """ValidateParticleIds (serialization.cpp:245-253) on the three particle populations."""
    for name, ids in (("Fluid", st.idF), ("Boundary", st.idB), ("Rigid", st.idR)):
        if ids.size and np.any(np.asarray(ids, np.uint64) == INVALID_PARTICLE_ID):
            raise SimStateError(f"{name} state contains the invalid particle ID sentinel.")


def _validate_attachments(st: UniversalSimState):
    """UniversalSimState::ValidateRigidAttachments (state_sim.h:679-713): every rigid particle
    names an existing body and the per-body counts equal the memberships."""
    if st.rigidParticleCountRB.size != st.N_RB:
        raise SimStateError("Invalid rigid body particle count array size.")
    body = np.asarray(st.bodyIdR, np.int64)
    if body.size and (body.min() < 0 or body.max() >= st.N_RB):
        raise SimStateError("Invalid rigid body index.")
    counts = np.bincount(body, minlength=st.N_RB) if st.N_RB else np.zeros(0, np.int64)
    if not np.array_equal(counts.astype(np.int64), np.asarray(st.rigidParticleCountRB, np.int64)):
        raise SimStateError("Rigid particle memberships do not match body counts.")


def _check_consistent(st: UniversalSimState):
    """Check*Consistent (serialization.cpp): every array has its population's length."""
    groups = ((st.N_F, ["idF"] + FLUID_F32), (st.N_B, ["idB"] + BOUNDARY_F32),
              (st.N_R, ["idR", "bodyIdR"] + RIGID_FIELDS), (st.N_RB, ["idRB", "rigidParticleCountRB"] + BODY_F32))
    for n, names in groups:
        for name in names:
            if np.asarray(getattr(st, name)).size != n:
                raise SimStateError(f"Array '{name}' does not match its population count {n}.")
    if st.N_RB and np.any(np.asarray(st.idRB, np.uint64) > U32_MAX):
        raise SimStateError("Rigid body ID exceeds the uint32 wire width.")


def save_universal_sim_state(st: UniversalSimState, path: str, atomic: bool = True,
                             temp_suffix: str = ".tmp"):
    """SaveUniversalSimState (serialization.cpp:838-885): validate the state (nothing is
    written when it fails), create the parent directory, write header + arrays; with `atomic`
    the file is written beside `path` and renamed over it."""
    _check_consistent(st)
    _validate_attachments(st)
    _validate_ids(st)
    compute_sim_state_offsets(st.N_F, st.N_B, st.N_R, st.N_RB)
    parent = os.path.dirname(os.path.abspath(path))
    os.makedirs(parent, exist_ok=True)
    tmp = path + temp_suffix if atomic else path
    try:
        _write_arrays(st, tmp)
    except BaseException:
        if atomic and os.path.exists(tmp):
            os.remove(tmp)
        raise
    if atomic:
        os.replace(tmp, path)


def _write_arrays(st: UniversalSimState, tmp: str):
    with open(tmp, "wb") as f:
        f.write(make_header(int(st.step), float(st.time), st.N_F, st.N_B, st.N_R, st.N_RB))
        f.write(np.asarray(st.idF, "<u8").tobytes())
        for n in FLUID_F32:
            f.write(np.asarray(getattr(st, n), "<f4").tobytes())
        f.write(np.asarray(st.idB, "<u8").tobytes())
        for n in BOUNDARY_F32:
            f.write(np.asarray(getattr(st, n), "<f4").tobytes())
        f.write(np.asarray(st.idR, "<u8").tobytes())
        f.write(np.asarray(st.bodyIdR, "<u4").tobytes())
        for n in RIGID_FIELDS:
            f.write(np.asarray(getattr(st, n), "<f4").tobytes())
        f.write(np.asarray(st.idRB, "<u4").tobytes())
        f.write(np.asarray(st.rigidParticleCountRB, "<u4").tobytes())
        for n in BODY_F32:
            f.write(np.asarray(getattr(st, n), "<f4").tobytes())


def load_universal_sim_state(path: str, into: UniversalSimState | None = None) -> UniversalSimState:
    """LoadUniversalSimState (serialization.cpp:887-935) with ReadSimStateHeader's checks
    (serialization.cpp:214-240): header tags, step/time, counts, exact file length; then the
    particle IDs and the rigid attachments. With `into`, that state's arrays and metadata are
    replaced (the reference's load-into-reference form) and it is returned."""
    size = os.path.getsize(path)
    with open(path, "rb") as f:
        raw = f.read(HEADER.size)
        if len(raw) != HEADER.size:
            raise SimStateError(f"Invalid simulation state header in '{path}'.")
        magic, tag, hbytes, step, time, n_f, n_b, n_r, n_rb = HEADER.unpack(raw)
        if magic != MAGIC or tag != ENDIAN_TAG or hbytes != HEADER.size:
            raise SimStateError(f"Invalid simulation state header in '{path}'.")
        if not math.isfinite(time) or time < 0.0 or step == U64_MAX:
            raise SimStateError("Invalid simulation state step/time.")
        if n_rb > U32_MAX:
            raise SimStateError("Serialized rigid body count exceeds uint32_t range.")
        off = compute_sim_state_offsets(n_f, n_b, n_r, n_rb)
        if size != off["totalBytes"]:
            raise SimStateError(f"Simulation state file length does not match its header in '{path}'.")
        for name, n in (("fluid", n_f), ("boundary", n_b), ("rigid", n_r)):
            if n > MAX_LOCAL_PARTICLE_COUNT:
                raise SimStateError(f"serialized {name} state exceeds the local particle limit.")
        data = f.read()
    st = UniversalSimState(n_f, n_b, n_r, n_rb)
    st.step, st.time = int(step), float(time)
    at = 0

    def take(n, dtype):
        nonlocal at
        dt = np.dtype(dtype)
        a = np.frombuffer(data, dt, n, at).copy()
        at += n * dt.itemsize
        return a

    st.idF = take(n_f, "<u8").astype(np.uint64)
    for n in FLUID_F32:
        setattr(st, n, take(n_f, "<f4").astype(np.float32))
    st.idB = take(n_b, "<u8").astype(np.uint64)
    for n in BOUNDARY_F32:
        setattr(st, n, take(n_b, "<f4").astype(np.float32))
    st.idR = take(n_r, "<u8").astype(np.uint64)
    st.bodyIdR = take(n_r, "<u4").astype(np.uint32)
    for n in RIGID_FIELDS:
        setattr(st, n, take(n_r, "<f4").astype(np.float32))
    st.idRB = take(n_rb, "<u4").astype(np.uint64)
    st.rigidParticleCountRB = take(n_rb, "<u4").astype(np.uint32)
    for n in BODY_F32:
        setattr(st, n, take(n_rb, "<f4").astype(np.float32))
    _validate_ids(st)
    _validate_attachments(st)
    if into is not None:
        into.__dict__.clear()
        into.__dict__.update(st.__dict__)
        return into
    return st
