"""GPU friends-of-friends (psod_fof through the C-ABI) against the oracle's
restatement of pFoF (oracle/psod_oracle_fof.c).

Exact: the halo member sets (the partition into groups of at least Mmin),
masses and counts; every halo's ID is the ID of its lowest-index member and
halos come in ascending ID.  The reference's own labels (the seed of its
sequential scan) differ by design; the oracle's are checked to name a member
of the same group.  Centres of mass agree within 1e-12 box units modulo the
box (FP64 sums in another order; the exact sums of most halos agree bit for
bit), radii within 1e-12, mean velocities within 1e-9 relative.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from psod_b200 import synth  # noqa: E402
from psod_b200.sod import PsodError, SphericalOverdensity  # noqa: E402

COM_ATOL = 1e-12
RAD_ATOL = 1e-12
VEL_RTOL = 1e-9


def gpu_fof(nx, pos, ids, vel=None, **kw):
    s = SphericalOverdensity(nx)
    s.load(pos, ids, vel=vel)
    st = s.fof(**kw)
    t = s.fof_halos()
    s.close()
    return st, t


def compare(t, r, pos, ids, vel):
    assert t.nhalo == r.nhalo
    assert int(t.member_offset[-1]) == int(r.member_offset[-1])
    gpu = {frozenset(t.members(h).tolist()): h for h in range(t.nhalo)}
    ora = {frozenset(r.members(h).tolist()): h for h in range(r.nhalo)}
    assert set(gpu) == set(ora)
    assert np.all(np.diff(t.halo_id) > 0)
    for m, h in gpu.items():
        q = ora[m]
        mem = t.members(h)
        assert np.all(np.diff(mem) > 0)  # ascending input index
        assert t.halo_id[h] == ids[mem.min()]
        assert r.halo_id[q] in set(ids[list(m)].tolist())
        assert t.halo_mass[h] == r.halo_mass[q] == len(m)
        d = np.abs(t.halo_com[h] - r.halo_com[q])
        d = np.minimum(d, np.abs(1.0 - d))
        assert np.all(d <= COM_ATOL), (h, t.halo_com[h], r.halo_com[q])
        assert abs(t.halo_radius[h] - r.halo_radius[q]) <= RAD_ATOL
        if vel is not None:
            assert np.allclose(t.halo_vel[h], r.halo_vel[q], rtol=VEL_RTOL, atol=1e-9)
    assert np.array_equal(t.member_id, ids[t.member_index])


@pytest.mark.parametrize("nx,mmin", [(32, 20), (48, 20), (64, 20), (64, 2)])
def test_fof_matches_oracle(oracle, nx, mmin):
    box = synth.make_box(nx, seed=77 + nx, nmax_halo=4000)
    pos = box.pos.numpy()
    ids = box.ids.numpy()
    vel = np.random.default_rng(nx).normal(0, 300, pos.shape).astype(np.float32)
    st, t = gpu_fof(nx, box.pos, box.ids, vel=torch.from_numpy(vel), percolation=0.2, mmin=mmin)
    r = oracle.fof(pos, ids, vel=vel, percolation=0.2, nres=nx, mmin=mmin)
    assert r.status == 0
    compare(t, r, pos, ids, vel)
    assert st["nhalo"] == t.nhalo
    assert st["ngroups"] == len(set(r.structure.tolist()))


def test_fof_uniform_box_with_bridges(oracle):
    nx = 40
    rng = np.random.default_rng(11)
    pos = rng.random((nx ** 3, 3), dtype=np.float32)
    # a few groups straddling every face and the corner
    for k, c in enumerate([(0.0005, 0.5, 0.5), (0.5, 0.9998, 0.5), (0.5, 0.5, 0.0001), (0.9999, 0.0002, 0.9997)]):
        pts = (np.array(c) + rng.normal(0, 0.0015, (30, 3))) % 1.0
        pos[k * 30:(k + 1) * 30] = pts.astype(np.float32)
    pos[pos >= 1.0] = 0.0
    ids = rng.permutation(len(pos)).astype(np.int64) + 1000
    st, t = gpu_fof(nx, torch.from_numpy(pos), torch.from_numpy(ids), percolation=0.2, mmin=2)
    r = oracle.fof(pos, ids, percolation=0.2, nres=nx, mmin=2)
    assert r.nbridges > 0
    compare(t, r, pos, ids, None)


def test_fof_config_box_128(oracle):
    """The 128^3 box of the CPU-runnable configuration (2,097,152 particles,
    halo N in [20, 2e4], b = 0.2, 20-particle minimum)."""
    box = synth.make_box(128, nmax_halo=20000)
    pos = box.pos.numpy()
    ids = box.ids.numpy()
    st, t = gpu_fof(128, box.pos, box.ids, percolation=0.2, mmin=20)
    r = oracle.fof(pos, ids, percolation=0.2, nres=128, mmin=20)
    compare(t, r, pos, ids, None)
    assert t.nhalo > 1000


def test_fof_runs_twice_and_after_sod(oracle):
    box = synth.make_box(32, seed=5, nmax_halo=3000)
    s = SphericalOverdensity(32)
    s.load(box.pos, box.ids)
    s.fof(percolation=0.2, mmin=20)
    a = s.fof_halos()
    s.run()
    s.fof(percolation=0.2, mmin=20)
    b = s.fof_halos()
    s.close()
    assert np.array_equal(a.halo_id, b.halo_id) and np.array_equal(a.member_index, b.member_index)
    assert np.array_equal(a.halo_com, b.halo_com) and np.array_equal(a.halo_radius, b.halo_radius)


def test_fof_arguments():
    box = synth.make_box(16, seed=3, nmax_halo=500)
    s = SphericalOverdensity(16)
    with pytest.raises(PsodError):
        s.fof_halos()  # no catalogue yet
    s.load(box.pos, box.ids)
    with pytest.raises(PsodError):
        s.fof(percolation=0.5)
    with pytest.raises(PsodError):
        s.fof(percolation=0.2, mmin=0)
    s.close()
