"""The reference's zone decomposition (main:321-441, 573-600, 2118-2120,
2370): zone selection, the rank -> zone assignment, the P-zone oracle on
known answers, the host logic over two gloo ranks, and (on a GPU) each zone
of the engine bit-exact against the oracle's zone run."""

import os
import socket
import sys

import numpy as np
import pytest

from tests.boxes import hole_ball_box

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_select_zone_matches_oracle(oracle):
    """psod_select_zone (host code of the library) keeps exactly the
    particles the oracle's restatement of main:573-600 keeps, including
    positions on zone and buffer edges."""
    from psod_b200.sod import select_zone

    rng = np.random.default_rng(5)
    for nx, nxcpu, nxb in ((32, 1, 0), (32, 2, 0), (48, 3, 0), (48, 3, 5), (64, 4, 0), (64, 4, 16)):
        edges = np.arange(0, nx + 1, dtype=np.float64) / nx
        ed = np.concatenate([edges, np.nextafter(edges.astype(np.float32), np.float32(2)),
                             np.nextafter(edges.astype(np.float32), np.float32(-1))]).astype(np.float32)
        ed = ed[(ed >= 0) & (ed < 1)]
        pos = rng.random((4000, 3)).astype(np.float32)
        m = len(ed) // 3
        pos[:m] = ed[: 3 * m].reshape(-1, 3)
        pos = np.concatenate([pos, np.stack([ed, ed, ed], 1)], 0)
        for z in range(nxcpu ** 3):
            a = select_zone(pos, nx, nxcpu, z, nxb)
            b = oracle.zone_select(pos, nx, nxcpu, z, nxb)
            assert np.array_equal(a, b), (nx, nxcpu, nxb, z)


def test_zones_of_rank_partition():
    """main:321-331: every zone goes to exactly one rank, in order, and the
    first nzones mod nranks ranks take one zone more."""
    from psod_b200.zones import zones_of_rank

    for nzones in (1, 8, 27, 64, 125):
        for nranks in (1, 2, 3, 5, 8, 16):
            got = [list(zones_of_rank(r, nranks, nzones)) for r in range(nranks)]
            assert sum(got, []) == list(range(nzones))
            sizes = [len(g) for g in got]
            nmod = nzones % nranks
            assert sizes == [nzones // nranks + (1 if r < nmod else 0) for r in range(nranks)]


def _lattice_ball_box(nx, centre):
    return hole_ball_box(nx, [centre], r_hole=3.6, r_ball=0.3, seed=9)


def test_oracle_zone_known_answer(oracle):
    """A compact ball in a lattice hole lies inside one zone of 4^3: that
    zone alone reports it (N_200 = the ball, members = the ball); the zones
    whose buffer holds it process it and reject it (main:2118-2120), and the
    lattice gives no other halo."""
    nx, nxcpu = 64, 4
    centre = (40.3, 9.7, 25.2)  # zone (2, 0, 1): nzone = 2*16 + 0*4 + 1 = 33
    pos, ids, balls = _lattice_ball_box(nx, centre)
    n = pos.shape[0]
    found = {}
    for z in range(nxcpu ** 3):
        k = oracle.zone_select(pos, nx, nxcpu, z)
        sel = np.nonzero(k)[0]
        r = oracle.run(oracle.Params(nx=nx, nxcpu=nxcpu, nzone=z, npart_total=n), pos[sel], ids[sel], oracle.CANONICAL)
        assert r.status == 0
        if r.nhalo:
            found[z] = (r, sel)
    assert list(found) == [33]
    r, sel = found[33]
    assert r.nhalo == 1 and r.halo_mass[0] == len(balls[0])
    assert np.array_equal(np.sort(sel[r.member_index]), balls[0])


def test_oracle_zones_equal_one_zone_on_a_clustered_box(oracle):
    """With a buffer wider than every halo, the zones' catalogues together
    are the one-zone catalogue (48^3 clustered box, 27 zones; 2^3 zones,
    whose buffers span the box, give it too)."""
    from psod_b200 import synth

    b = synth.make_box(48, nmax_halo=4000, seed=11)
    pos, ids = b.pos.numpy(), b.ids.numpy()
    n = pos.shape[0]
    one = oracle.run(oracle.Params(nx=48), pos, ids, oracle.CANONICAL)
    ref = {int(i): int(m) for i, m in zip(one.halo_id, one.halo_mass)}
    for nxcpu in (2, 3):
        got = {}
        for z in range(nxcpu ** 3):
            k = oracle.zone_select(pos, 48, nxcpu, z)
            r = oracle.run(oracle.Params(nx=48, nxcpu=nxcpu, nzone=z, npart_total=n), pos[k], ids[k],
                           oracle.CANONICAL)
            assert r.status == 0
            for i, m in zip(r.halo_id, r.halo_mass):
                assert int(i) not in got
                got[int(i)] = int(m)
        assert got == ref, nxcpu


def test_zone_parameters_refused():
    """Zone parameters are checked before any device work: nx a multiple of
    nxcpu, nzone in range, nxbuffer <= nxzone, and no local grid just short
    of the box (its wrapped cell walks would reach its far side)."""
    import ctypes as C

    from psod_b200 import capi

    lib = capi.load()
    for kw in (dict(nx=32, nxcpu=3), dict(nx=32, nxcpu=2, nzone=8), dict(nx=32, nxcpu=2, nzone=-1),
               dict(nx=32, nxcpu=2, nxbuffer=17), dict(nx=48, nxcpu=2, nxbuffer=11, ncut=4)):
        p = capi.default_params(**kw)
        h = C.c_void_p()
        assert lib.psod_ctx_create(C.byref(p), C.byref(h)) == capi.ERR_ARG, kw


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from oracle import oracle as O
    from psod_b200 import synth
    from psod_b200.zones import run_zones

    dist.init_process_group("gloo", rank=rank, world_size=world)
    b = synth.make_box(32, nmax_halo=2000, seed=7)
    pos, ids = b.pos.numpy(), b.ids.numpy()

    def run_zone(p, i, z):  # the oracle as the zone runner (CPU)
        k = O.zone_select(p, 32, 2, z)
        return O.run(O.Params(nx=32, nxcpu=2, nzone=z, npart_total=p.shape[0]), p[k], i[k], O.CANONICAL)

    tables, total = run_zones(pos, ids, 2, run_zone, rank=rank, nranks=world)
    q.put((rank, sorted(tables), sum(t.nhalo for t in tables.values()), total))
    dist.destroy_process_group()


def test_two_ranks_over_gloo(oracle):
    """Two ranks split the 8 zones (0-3, 4-7) and all-reduce their halo
    counts; the total equals one process running every zone."""
    pytest.importorskip("torch")
    import torch.multiprocessing as mp

    from psod_b200 import synth
    from psod_b200.zones import run_zones

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert [o[1] for o in out] == [[0, 1, 2, 3], [4, 5, 6, 7]]
    b = synth.make_box(32, nmax_halo=2000, seed=7)
    pos, ids = b.pos.numpy(), b.ids.numpy()

    def run_zone(p, i, z):
        k = oracle.zone_select(p, 32, 2, z)
        return oracle.run(oracle.Params(nx=32, nxcpu=2, nzone=z, npart_total=p.shape[0]), p[k], i[k],
                          oracle.CANONICAL)

    _, single = run_zones(pos, ids, 2, run_zone)
    assert out[0][3] == out[1][3] == single == out[0][2] + out[1][2]


# ---------------------------------------------------------------------------
# GPU: each zone of the engine against the oracle's zone run
# ---------------------------------------------------------------------------
def _gpu_or_skip():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("nx,nxcpu,nmax", [(32, 2, 2000), (48, 3, 4000)])
@pytest.mark.parametrize("mode", [0, 1])
def test_gpu_zones_match_oracle(oracle, nx, nxcpu, nmax, mode):
    """Every zone (2^3 of a 32^3 box, 3^3 of a 48^3 box), plain and batched:
    rho, the seed order and the halo table (IDs, masses, ranks, centres,
    R_delta, member lists in order) bit-exact against the oracle's canonical
    zone run on the same selected particles."""
    torch = _gpu_or_skip()
    from psod_b200 import synth
    from psod_b200.sod import SphericalOverdensity, select_zone

    b = synth.make_box(nx, nmax_halo=nmax, seed=11)
    pos, ids = b.pos.numpy(), b.ids.numpy()
    n = pos.shape[0]
    total = 0
    for z in range(nxcpu ** 3):
        sel = np.nonzero(select_zone(pos, nx, nxcpu, z))[0]
        p, i = np.ascontiguousarray(pos[sel]), np.ascontiguousarray(ids[sel])
        op = oracle.Params(nx=nx, nxcpu=nxcpu, nzone=z, npart_total=n)
        r = oracle.run(op, p, i, oracle.CANONICAL)
        rho_o = oracle.rho(op, p, oracle.CANONICAL)
        with SphericalOverdensity(nx, device=0, nxcpu=nxcpu, nzone=z, mode=mode) as s:
            s.load(torch.from_numpy(p).cuda(), torch.from_numpy(i).cuda(), npart_total=n)
            s.cic()
            rho = s.cicm1()
            isort, nn = s.tri_cic()
            s.spherover()
            t = s.halos()
        assert np.array_equal(rho, rho_o), z
        iso, nno = oracle.tri_cic(rho_o, oracle.CANONICAL)
        assert nn == nno == r.npart_new and np.array_equal(isort[:nn], iso[:nn]), z
        assert t.nhalo == r.nhalo, z
        for f in ("halo_id", "halo_mass", "halo_rank", "halo_center", "halo_rdelta", "member_offset",
                  "member_index"):
            assert np.array_equal(getattr(t, f), getattr(r, f)), (z, f)
        total += t.nhalo
    assert total > 0


@pytest.mark.gpu
def test_gpu_zone_runner_and_count(oracle):
    """psod_b200.zones on one GPU: every zone of the 32^3 box through the
    GPU zone runner; the tables (member indices back in the full particle
    arrays) and the summed count equal the oracle's zone runs."""
    _gpu_or_skip()
    from psod_b200 import synth
    from psod_b200.zones import gpu_zone_runner, run_zones

    b = synth.make_box(32, nmax_halo=2000, seed=11)
    pos, ids = b.pos.numpy(), b.ids.numpy()
    n = pos.shape[0]
    tables, count = run_zones(pos, ids, 2, gpu_zone_runner(32, 2, mode=1))
    total = 0
    for z, t in tables.items():
        sel = np.nonzero(oracle.zone_select(pos, 32, 2, z))[0]
        r = oracle.run(oracle.Params(nx=32, nxcpu=2, nzone=z, npart_total=n), pos[sel], ids[sel], oracle.CANONICAL)
        assert np.array_equal(t.halo_id, r.halo_id) and np.array_equal(t.halo_mass, r.halo_mass), z
        assert np.array_equal(t.member_index, sel[r.member_index]), z
        total += r.nhalo
    assert count == total > 0


def test_oracle_refuses_the_same_zone_parameters(oracle):
    """The oracle's zone set-up refuses what psod_ctx_create refuses: nx not
    a multiple of nxcpu, nzone out of range, a buffer wider than the zone,
    and a local grid just short of the box."""
    pos = np.random.default_rng(1).random((1000, 3)).astype(np.float32)
    ids = np.arange(1000, dtype=np.int64)
    for kw in (dict(nx=32, nxcpu=3), dict(nx=32, nxcpu=2, nzone=8), dict(nx=32, nxcpu=2, nxbuffer=17),
               dict(nx=48, nxcpu=2, nxbuffer=11, ncut=4)):
        r = oracle.run(oracle.Params(npart_total=1000, **kw), pos, ids, oracle.CANONICAL)
        assert r.status != 0, kw
    r = oracle.run(oracle.Params(nx=48, nxcpu=3, nzone=13, npart_total=1000), pos, ids, oracle.CANONICAL)
    assert r.status == 0
