"""TSPSIM2 state files: the reference's known layout and rejection cases
(tests/unit/state_serialization.cpp), rebuilt here from an independent byte encoder."""
import math
import struct

import numpy as np
import pytest

from turbospharticles_b200.state import BODY_F32, BOUNDARY_F32, FLUID_F32, UniversalSimState
from turbospharticles_b200.state_io import (SimStateError, compute_sim_state_offsets, load_universal_sim_state,
                                            save_universal_sim_state)

RIGID_FILE_F32 = ["xPosRelR", "yPosRelR", "zPosRelR", "volR", "psiR"]
U64_MAX = (1 << 64) - 1


def fill(st, names, base):
    for f, name in enumerate(names):
        a = getattr(st, name)
        a[:] = base + np.arange(a.size, dtype=np.float32) + np.float32(16 * f) + np.float32(0.25)


def make_state(n_f=2, n_b=1, n_r=3, n_rb=2):
    """The reference test's mixed state: distinct values in every field, wide IDs, signed zero."""
    st = UniversalSimState(n_f, n_b, n_r, n_rb)
    st.step, st.time = 0x0102030405060708, 12.5
    fill(st, FLUID_F32, np.float32(100.0))
    fill(st, BOUNDARY_F32, np.float32(1000.0))
    fill(st, RIGID_FILE_F32, np.float32(2000.0))
    fill(st, BODY_F32, np.float32(3000.0))
    st.idF[:] = 5_000_000_000 + 17 * np.arange(n_f, dtype=np.uint64)
    st.idB[:] = 6_000_000_000 + 19 * np.arange(n_b, dtype=np.uint64)
    st.idRB[:] = 100 + 7 * np.arange(n_rb, dtype=np.uint64)
    st.rigidParticleCountRB[:] = 0
    for i in range(n_r):
        st.idR[i] = 7_000_000_000 + 23 * i
        st.bodyIdR[i] = i % n_rb
        st.rigidParticleCountRB[i % n_rb] += 1
    if n_f:
        st.idF[0] = U64_MAX - 1
        st.yVelF[0] = -123.5
        st.zVelF[0] = -0.0
    return st


def expected_bytes(st):
    """Byte-by-byte encoding of the documented layout, independent of the writer."""
    b = bytearray(b"TSPSIM2\x00" + bytes([4, 3, 2, 1, 64, 0, 0, 0]))
    b += struct.pack("<Q", st.step) + struct.pack("<d", st.time)
    for n in (st.N_F, st.N_B, st.N_R, st.N_RB):
        b += struct.pack("<Q", n)

    def put(values, fmt):
        nonlocal b
        for v in values:
            b += struct.pack("<" + fmt, v.item() if hasattr(v, "item") else v)

    put(st.idF, "Q")
    for n in FLUID_F32:
        put(getattr(st, n), "f")
    put(st.idB, "Q")
    for n in BOUNDARY_F32:
        put(getattr(st, n), "f")
    put(st.idR, "Q")
    put(st.bodyIdR, "I")
    for n in RIGID_FILE_F32:
        put(getattr(st, n), "f")
    put(st.idRB, "I")
    put(st.rigidParticleCountRB, "I")
    for n in BODY_F32:
        put(getattr(st, n), "f")
    return bytes(b)


def assert_state_equal(a, e):
    assert (a.step, a.N_F, a.N_B, a.N_R, a.N_RB) == (e.step, e.N_F, e.N_B, e.N_R, e.N_RB)
    assert struct.pack("<d", a.time) == struct.pack("<d", e.time)
    for n in ("idF", "idB", "idR", "bodyIdR", "idRB", "rigidParticleCountRB"):
        np.testing.assert_array_equal(np.asarray(getattr(a, n), np.uint64), np.asarray(getattr(e, n), np.uint64), n)
    for n in FLUID_F32 + BOUNDARY_F32 + RIGID_FILE_F32 + BODY_F32:  # bitwise: keeps -0.0 and every payload bit
        np.testing.assert_array_equal(getattr(a, n).view(np.uint32), getattr(e, n).view(np.uint32), n)


def test_round_trips_every_state_field(tmp_path):
    e = make_state()
    save_universal_sim_state(e, str(tmp_path / "state.bin"))
    assert_state_equal(load_universal_sim_state(str(tmp_path / "state.bin")), e)


def test_writes_expected_binary_layout(tmp_path):
    st = make_state()
    exp = expected_bytes(st)
    assert len(exp) == 604
    save_universal_sim_state(st, str(tmp_path / "state.bin"))
    assert (tmp_path / "state.bin").read_bytes() == exp
    assert not (tmp_path / "state.bin.tmp").exists()


def test_loads_independently_encoded_state(tmp_path):
    e = make_state()
    (tmp_path / "state.bin").write_bytes(expected_bytes(e))
    assert_state_equal(load_universal_sim_state(str(tmp_path / "state.bin")), e)


@pytest.mark.parametrize("counts", [(0, 0, 0, 0), (2, 0, 0, 0), (0, 2, 0, 0), (0, 0, 3, 2), (0, 1, 3, 2),
                                    (2, 0, 3, 2), (2, 1, 0, 0)])
def test_round_trips_empty_populations(tmp_path, counts):
    e = make_state(*counts)
    p = tmp_path / "state.bin"
    save_universal_sim_state(e, str(p))
    assert_state_equal(load_universal_sim_state(str(p)), e)
    n_f, n_b, n_r, n_rb = counts
    assert p.stat().st_size == 64 + 72 * n_f + 28 * n_b + 32 * n_r + 136 * n_rb


def test_replaces_previously_loaded_state(tmp_path):
    states = [make_state(5, 3, 4, 3), make_state(1, 0, 1, 1), make_state(0, 0, 0, 0), make_state()]
    actual = make_state(2, 2, 2, 2)
    for i, e in enumerate(states):
        e.step += i
        e.time += 0.125 * i
        save_universal_sim_state(e, str(tmp_path / "state.bin"))
        got = load_universal_sim_state(str(tmp_path / "state.bin"), into=actual)
        assert got is actual
        assert_state_equal(actual, e)


def _load_bytes(tmp_path, data):
    (tmp_path / "state.bin").write_bytes(bytes(data))
    return load_universal_sim_state(str(tmp_path / "state.bin"))


@pytest.mark.parametrize("length", [0, 1, 63])
def test_rejects_truncated_headers(tmp_path, length):
    with pytest.raises(SimStateError):
        _load_bytes(tmp_path, expected_bytes(make_state())[:length])


@pytest.mark.parametrize("offset", [0, 6, 7, 8, 12])
def test_rejects_invalid_header_tags(tmp_path, offset):
    b = bytearray(expected_bytes(make_state()))
    b[offset] ^= 0xFF
    with pytest.raises(SimStateError):
        _load_bytes(tmp_path, b)


@pytest.mark.parametrize("offset", [32, 40, 48, 56])
def test_rejects_mismatched_population_counts(tmp_path, offset):
    b = bytearray(expected_bytes(make_state()))
    b[offset] += 1
    with pytest.raises(SimStateError):
        _load_bytes(tmp_path, b)


@pytest.mark.parametrize("length", [64, 208, 603, 605])
def test_rejects_incorrect_payload_lengths(tmp_path, length):
    b = bytearray(expected_bytes(make_state()))
    b = b[:length] if length <= len(b) else b + bytes(length - len(b))
    with pytest.raises(SimStateError):
        _load_bytes(tmp_path, b)


@pytest.mark.parametrize("time", [-1.0, math.inf, math.nan])
def test_rejects_invalid_time(tmp_path, time):
    b = bytearray(expected_bytes(make_state()))
    b[24:32] = struct.pack("<d", time)
    with pytest.raises(SimStateError):
        _load_bytes(tmp_path, b)


def test_rejects_invalid_step(tmp_path):
    b = bytearray(expected_bytes(make_state()))
    b[16:24] = struct.pack("<Q", U64_MAX)
    with pytest.raises(SimStateError):
        _load_bytes(tmp_path, b)


@pytest.mark.parametrize("offset", [64, 208, 236])
def test_rejects_invalid_particle_ids(tmp_path, offset):
    b = bytearray(expected_bytes(make_state()))
    b[offset:offset + 8] = struct.pack("<Q", U64_MAX)
    with pytest.raises(SimStateError):
        _load_bytes(tmp_path, b)


@pytest.mark.parametrize("population", ["idF", "idB", "idR"])
def test_rejects_saving_invalid_particle_ids(tmp_path, population):
    st = make_state()
    getattr(st, population)[0] = np.uint64(U64_MAX)
    with pytest.raises(SimStateError):
        save_universal_sim_state(st, str(tmp_path / "state.bin"))
    assert not (tmp_path / "state.bin").exists()


def test_rejects_saving_out_of_range_rigid_body_indices(tmp_path):
    st = make_state()
    st.bodyIdR[0] = st.N_RB
    with pytest.raises(SimStateError):
        save_universal_sim_state(st, str(tmp_path / "state.bin"))
    assert not (tmp_path / "state.bin").exists()


def test_rejects_saving_mismatched_rigid_body_particle_counts(tmp_path):
    st = make_state()
    st.rigidParticleCountRB[0] -= 1
    with pytest.raises(SimStateError):
        save_universal_sim_state(st, str(tmp_path / "state.bin"))
    assert not (tmp_path / "state.bin").exists()


@pytest.mark.parametrize("offset,value", [(260, 2), (340, 1)])
def test_rejects_invalid_rigid_attachments(tmp_path, offset, value):
    """Offset 260 is the first rigid bodyId (set to a body that does not exist); 340 is the
    first body's particle count (no longer equal to its memberships)."""
    b = bytearray(expected_bytes(make_state()))
    b[offset] = value
    with pytest.raises(SimStateError):
        _load_bytes(tmp_path, b)


def test_computes_mixed_population_offsets():
    off = compute_sim_state_offsets(2, 1, 3, 2)
    assert (off["fluid"], off["boundary"], off["rigid"], off["rigidBodies"], off["totalBytes"]) == (64, 208, 236, 332, 604)


def test_empty_populations_contain_only_header():
    off = compute_sim_state_offsets(0, 0, 0, 0)
    assert set(off.values()) == {64}


def test_keeps_offsets_wider_than_32_bits():
    off = compute_sim_state_offsets(67_108_864, 0, 0, 0)
    assert off["fluid"] == 64
    assert off["boundary"] == off["rigid"] == off["rigidBodies"] == off["totalBytes"] == 4_831_838_272


@pytest.mark.parametrize("which", range(4))
def test_rejects_overflowing_offsets(which):
    counts = [0, 0, 0, 0]
    counts[which] = U64_MAX
    with pytest.raises(SimStateError):
        compute_sim_state_offsets(*counts)


def test_rejects_overflowing_header_plus_payload():
    with pytest.raises(SimStateError):
        compute_sim_state_offsets(U64_MAX // 72, 0, 0, 0)
