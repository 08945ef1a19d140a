"""The reference's binary particle reader (main:455-534): the cube files
"<root>_cube_NNNNN" (Fortran unformatted sequential records: nloc, rank,
bounds, positions, velocities, IDs) read through the C-ABI for one zone,
against a plain-Python restatement of the reference's file list (27 cubes
around the zone, x outer, z inner, periodic, main:363-375) and distance test
(main:471-479).  Host only, no GPU."""

import struct

import numpy as np
import pytest

from psod_b200 import capi
from psod_b200.sod import PsodError, read_cube_zone


def rec(payload: bytes, split: int = 0) -> bytes:
    """One Fortran record; split > 0 writes it as gfortran subrecords of
    that many bytes (negative leading marker while more follow)."""
    if split <= 0 or len(payload) <= split:
        return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))
    out = b""
    for k in range(0, len(payload), split):
        part = payload[k : k + split]
        more = k + split < len(payload)
        head = -len(part) if more else len(part)
        tail = len(part) if k == 0 else -len(part)
        out += struct.pack("<i", head) + part + struct.pack("<i", tail)
    return out


def write_cubes(root, ncpu, per_file, seed=1, id_bytes=8, split=0):
    """ncpu cube files with uniform particles inside each cube's bounds."""
    n = round(ncpu ** (1 / 3))
    rng = np.random.default_rng(seed)
    files = {}
    for f in range(ncpu):
        fi, fj, fk = f // (n * n), (f // n) % n, f % n
        lo = np.array([fi, fj, fk], np.float64) / n
        pos = (lo + rng.random((per_file, 3)) / n).astype(np.float32)
        pos = np.minimum(pos, np.float32(np.nextafter(np.float32(1), np.float32(0))))
        vel = rng.normal(size=(per_file, 3)).astype(np.float32)
        ids = (f * 1_000_000 + np.arange(per_file)).astype(np.int64 if id_bytes == 8 else np.int32)
        hi = lo + 1.0 / n
        body = rec(struct.pack("<i", per_file)) + rec(struct.pack("<i", f))
        body += rec(struct.pack("<6f", lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]))
        body += rec(pos.tobytes(), split) + rec(vel.tobytes(), split) + rec(ids.tobytes(), split)
        (root.parent / f"{root.name}_cube_{f:05d}").write_bytes(body)
        files[f] = (pos, vel, ids.astype(np.int64))
    return files


def reference_zone(files, ncpu, nzone, nx, nxbuffer):
    """main:340-439 and 455-534 in plain Python (each listed cube once)."""
    n = round(ncpu ** (1 / 3))
    ix = int(nzone / float(n * n))
    iy = int((nzone - ix * n * n) / float(n))
    iz = nzone - ix * n * n - iy * n
    nxzone = nx // n
    nxb = nxzone // 2 if nxbuffer == 0 else nxbuffer
    order = []
    for i in range(ix - 1, ix + 2):
        for j in range(iy - 1, iy + 2):
            for k in range(iz - 1, iz + 2):
                it, jt, kt = (n - 1 if i < 0 else i), (n - 1 if j < 0 else j), (n - 1 if k < 0 else k)
                f = kt % n + (jt % n) * n + (it % n) * n * n
                if f not in order:
                    order.append(f)
    c = [((a / n) + ((a + 1) / n)) / 2.0 for a in (ix, iy, iz)]
    rs = (0.5 + nxb / nxzone) / n
    rl = 1.0 - rs
    P, V, I = [], [], []
    for f in order:
        pos, vel, ids = files[f]
        for q in range(pos.shape[0]):
            ok = True
            for a in range(3):
                d = abs(float(pos[q, a]) - c[a])
                ok = ok and (d < rs or d > rl)
            if ok:
                P.append(pos[q]), V.append(vel[q]), I.append(ids[q])
    return np.array(P, np.float32).reshape(-1, 3), np.array(V, np.float32).reshape(-1, 3), np.array(I, np.int64)


@pytest.mark.parametrize("nzone", [0, 13, 26])
def test_zone_of_27_cubes(tmp_path, nzone):
    root = tmp_path / "fof"
    files = write_cubes(root, 27, 300, seed=nzone)
    pos, vel, ids = read_cube_zone(str(root), 27, nzone, nx=24, nxbuffer=0)
    rp, rv, ri = reference_zone(files, 27, nzone, 24, 0)
    assert ids.size == ri.size > 0
    assert np.array_equal(pos, rp) and np.array_equal(vel, rv) and np.array_equal(ids, ri)


def test_subrecords_int32_ids_and_buffer(tmp_path):
    root = tmp_path / "sim"
    files = write_cubes(root, 27, 200, seed=5, id_bytes=4, split=64)
    pos, vel, ids = read_cube_zone(str(root), 27, 4, nx=24, nxbuffer=3, id_bytes=4)
    rp, rv, ri = reference_zone(files, 27, 4, 24, 3)
    assert np.array_equal(pos, rp) and np.array_equal(vel, rv) and np.array_equal(ids, ri)


def test_single_cube_reads_each_particle_once(tmp_path, oracle):
    """One cube per side: the zone is the whole box.  The particles come back
    in file order and the oracle's SOD on them equals its SOD on the
    generator's arrays."""
    from psod_b200 import synth

    b = synth.make_box(16, nmax_halo=500, seed=9)
    p, i = b.pos.numpy(), b.ids.numpy()
    body = rec(struct.pack("<i", p.shape[0])) + rec(struct.pack("<i", 0)) + rec(struct.pack("<6f", 0, 1, 0, 1, 0, 1))
    body += rec(p.tobytes()) + rec(np.zeros_like(p).tobytes()) + rec(i.tobytes())
    (tmp_path / "one_cube_00000").write_bytes(body)
    pos, vel, ids = read_cube_zone(str(tmp_path / "one"), 1, 0, nx=16)
    assert np.array_equal(pos, p) and np.array_equal(ids, i)
    r1 = oracle.run(oracle.Params(nx=16, nmin=20), pos, ids, oracle.CANONICAL)
    r2 = oracle.run(oracle.Params(nx=16, nmin=20), p, i, oracle.CANONICAL)
    assert np.array_equal(r1.halo_id, r2.halo_id) and np.array_equal(r1.member_index, r2.member_index)


def test_reader_errors(tmp_path):
    import ctypes as C

    root = tmp_path / "x"
    write_cubes(root, 27, 50)
    with pytest.raises(PsodError) as e:
        read_cube_zone(str(tmp_path / "missing"), 27, 0, nx=24)
    assert e.value.status == capi.ERR_IO
    # a truncated file
    f = tmp_path / "x_cube_00013"
    f.write_bytes(f.read_bytes()[:-10])
    with pytest.raises(PsodError) as e:
        read_cube_zone(str(root), 27, 13, nx=24)
    assert e.value.status == capi.ERR_IO
    lib = capi.load()
    n = C.c_int64(0)
    # ncpu not a cube, zone out of range, buffer wider than the zone
    for args in ((26, 0, 24, 0), (27, 27, 24, 0), (27, 0, 24, 9)):
        assert lib.psod_read_cube_zone(str(root).encode(), *args, 8, 0, C.byref(n), None, None, None) == capi.ERR_ARG
    # a capacity below the zone's count
    write_cubes(root, 27, 50)
    assert lib.psod_read_cube_zone(str(root).encode(), 27, 0, 24, 0, 8, 0, C.byref(n), None, None, None) == capi.OK
    buf = np.zeros((n.value, 3), np.float32)
    idb = np.zeros(n.value, np.int64)
    st = lib.psod_read_cube_zone(str(root).encode(), 27, 0, 24, 0, 8, n.value - 1, C.byref(n),
                                 C.c_void_p(buf.ctypes.data), None, C.c_void_p(idb.ctypes.data))
    assert st == capi.ERR_ARG
