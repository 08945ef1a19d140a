"""The reference's binary halo files (main:2230-2259) from the halo table:
Fortran unformatted sequential records, written by the C-ABI on the host
(no GPU needed).  Checked byte for byte on a hand-built table and record by
record against the oracle's halos on a clustered box."""

import struct

import numpy as np
import pytest

from psod_b200 import capi
from psod_b200.sod import HaloTable, PsodError, write_masst, write_strct


def records(path):
    """Split a Fortran unformatted sequential file into its record payloads
    (int32 length, payload, int32 length)."""
    out = []
    data = open(path, "rb").read()
    i = 0
    while i < len(data):
        (n,) = struct.unpack_from("<i", data, i)
        out.append(data[i + 4 : i + 4 + n])
        (m,) = struct.unpack_from("<i", data, i + 4 + n)
        assert m == n
        i += 8 + n
    return out


def table(halo_id, halo_mass, halo_center, member_offset, member_index):
    h = len(halo_id)
    return HaloTable(
        halo_id=np.asarray(halo_id, np.int64), halo_mass=np.asarray(halo_mass, np.int64),
        halo_rank=np.zeros(h, np.int64), halo_center=np.asarray(halo_center, np.float32).reshape(h, 3),
        halo_rdelta=np.zeros(h), halo_mass2=np.zeros(h, np.int64), halo_mextra=np.zeros((h, 0), np.int64),
        halo_profile=np.zeros((h, 0), np.int64), member_offset=np.asarray(member_offset, np.int64),
        member_index=np.asarray(member_index, np.int64), member_id=np.zeros(len(member_index), np.int64))


def test_bytes_of_a_small_table(tmp_path):
    pos = np.arange(15, dtype=np.float32).reshape(5, 3) / 16
    vel = -np.arange(15, dtype=np.float32).reshape(5, 3)
    ids = np.array([100, 101, 102, 103, 104], np.int64)
    t = table([102, 100], [2, 1], [[0.5, 0.25, 0.125], [0.75, 0.5, 0.0625]], [0, 2, 3], [2, 4, 0])
    write_masst(tmp_path / "m", t)
    rec = lambda b: struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))  # noqa: E731
    want = rec(struct.pack("<i", 2))
    want += rec(struct.pack("<qi3f", 102, 2, 0.5, 0.25, 0.125))
    want += rec(struct.pack("<qi3f", 100, 1, 0.75, 0.5, 0.0625))
    assert open(tmp_path / "m", "rb").read() == want
    write_strct(tmp_path / "s", t, pos, ids, vel=vel)
    want = rec(struct.pack("<i", 2))
    for members in ([2, 4], [0]):
        want += rec(struct.pack("<i", len(members)))
        want += rec(pos[members].tobytes())
        want += rec(vel[members].tobytes())
        want += rec(ids[members].tobytes())
    assert open(tmp_path / "s", "rb").read() == want
    # without velocities the reference's velf would be written; here zeros,
    # plus the optional potential and force records
    pot = np.arange(5, dtype=np.float32)
    force = np.ones((5, 3), np.float32)
    write_strct(tmp_path / "s2", t, pos, ids, pot=pot, force=force)
    r = records(tmp_path / "s2")
    assert len(r) == 1 + 2 * 6
    assert r[3] == np.zeros(6, np.float32).tobytes()
    assert r[5] == pot[[2, 4]].tobytes() and r[6] == force[[2, 4]].tobytes()


def test_oracle_halos_round_trip(oracle, tmp_path):
    from psod_b200 import synth

    b = synth.make_box(32, nmax_halo=2000, seed=123)
    pos, ids = b.pos.numpy(), b.ids.numpy()
    r = oracle.run(oracle.Params(nx=32), pos, ids, oracle.CANONICAL)
    assert r.status == 0 and r.nhalo > 10
    t = table(r.halo_id, r.halo_mass, r.halo_center, r.member_offset, r.member_index)
    vel = np.random.default_rng(1).normal(size=pos.shape).astype(np.float32)
    write_masst(tmp_path / "sod_00001_masst_00000", t)
    write_strct(tmp_path / "sod_00001_strct_00000", t, pos, ids, vel=vel)
    m = records(tmp_path / "sod_00001_masst_00000")
    assert struct.unpack("<i", m[0])[0] == r.nhalo and len(m) == 1 + r.nhalo
    for h in range(r.nhalo):
        hid, mass, x, y, z = struct.unpack("<qi3f", m[1 + h])
        assert hid == r.halo_id[h] and mass == r.halo_mass[h]
        assert np.array_equal(np.array([x, y, z], np.float32), r.halo_center[h])
    s = records(tmp_path / "sod_00001_strct_00000")
    assert struct.unpack("<i", s[0])[0] == r.nhalo and len(s) == 1 + 4 * r.nhalo
    for h in range(r.nhalo):
        mem = r.member_index[r.member_offset[h] : r.member_offset[h + 1]]
        assert struct.unpack("<i", s[1 + 4 * h])[0] == mem.size
        assert np.array_equal(np.frombuffer(s[2 + 4 * h], np.float32).reshape(-1, 3), pos[mem])
        assert np.array_equal(np.frombuffer(s[3 + 4 * h], np.float32).reshape(-1, 3), vel[mem])
        assert np.array_equal(np.frombuffer(s[4 + 4 * h], np.int64), ids[mem])


def test_writer_errors(tmp_path):
    pos = np.zeros((3, 3), np.float32)
    ids = np.arange(3, dtype=np.int64)
    t = table([0], [2], [[0, 0, 0]], [0, 2], [0, 7])  # member index beyond n
    with pytest.raises(PsodError) as e:
        write_strct(tmp_path / "s", t, pos, ids)
    assert e.value.status == capi.ERR_ARG
    # the table is checked before the file is opened: nothing is left behind
    assert not (tmp_path / "s").exists()
    t = table([0, 1], [1, -3], [[0, 0, 0], [0, 0, 0]], [0, 1, 1], [0])  # negative mass in the last record
    with pytest.raises(PsodError) as e:
        write_masst(tmp_path / "m_bad", t)
    assert e.value.status == capi.ERR_ARG
    assert not (tmp_path / "m_bad").exists()
    t = table([0], [2], [[0, 0, 0]], [0, 2], [0, 1])
    with pytest.raises(PsodError) as e:
        write_masst(tmp_path / "missing_dir" / "m", t)
    assert e.value.status == capi.ERR_IO
