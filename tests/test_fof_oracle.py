"""The friends-of-friends oracle (oracle/psod_oracle_fof.c) against known
answers and an independent periodic FoF (scipy's KD-tree with a periodic
box plus connected components).

pFoF ships no golden outputs, so these boxes pin the restatement:
  - friendship at the linking length, chains, the queue labels of the
    sequential scan (modfofpara.f90:158-288) and their merge to the smallest
    label across the periodic boundary (modfofmpi.f90:323-649);
  - bridges across each face and a corner (modfofmpi.f90:183-317);
  - Mmin, ascending labels and heap order (sod/modhalo.f90:253-376,
    modsortinterf.f90:650-681);
  - computecom's unwrap against the running mean and computeradius's
    periodic rule (sod/modhalo.f90:381-488).
"""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def _box(points):
    return np.asarray(points, np.float32).reshape(-1, 3)


def _groups(r):
    """partition as a set of frozensets of input indices (all particles)"""
    out = {}
    for i, s in enumerate(r.structure):
        out.setdefault(int(s), set()).add(i)
    return {frozenset(v) for v in out.values()}


def _brute_groups(pos, link):
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from scipy.spatial import cKDTree

    n = len(pos)
    pr = cKDTree(pos.astype(np.float64), boxsize=1.0).query_pairs(link, output_type="ndarray")
    g = coo_matrix((np.ones(len(pr)), (pr[:, 0], pr[:, 1])), shape=(n, n))
    lab = connected_components(g, directed=False)[1]
    out = {}
    for i, s in enumerate(lab):
        out.setdefault(int(s), set()).add(i)
    return {frozenset(v) for v in out.values()}


def test_pair_at_linking_length():
    # nres 10: linking length 0.02 box units
    pos = _box([[0.50, 0.5, 0.5], [0.515, 0.5, 0.5], [0.56, 0.5, 0.5]])
    r = O.fof(pos, np.array([7, 8, 9]), percolation=0.2, nres=10, mmin=1)
    assert r.status == 0
    assert _groups(r) == {frozenset({0, 1}), frozenset({2})}
    assert list(r.halo_mass) == [2, 1] and list(r.halo_id) == [7, 9]


def test_chain_is_one_group():
    x = 0.3 + 0.015 * np.arange(6)
    pos = _box([[v, 0.4, 0.4] for v in x])
    r = O.fof(pos, np.arange(1, 7), percolation=0.2, nres=10, mmin=1)
    assert _groups(r) == {frozenset(range(6))}
    assert r.nhalo == 1 and r.halo_mass[0] == 6


def test_queue_label_is_the_scan_seed_not_the_lowest_index():
    # particles 1-5 (1-based): 1~5 and 2~3 are friends.  The scan starts at 1,
    # finds 5, which takes the queue's front slot (particle 2 moves to slot
    # 5); the next group starts at the front slot 3, finds 2: that group is
    # labelled with particle 3's ID, not particle 2's.
    link = 0.02
    pos = _box([[0.1, 0.1, 0.1], [0.5, 0.5, 0.5], [0.5 + 0.5 * link, 0.5, 0.5], [0.8, 0.2, 0.3],
                [0.1 + 0.5 * link, 0.1, 0.1]])
    ids = np.array([1, 2, 3, 4, 5])
    r = O.fof(pos, ids, percolation=0.2, nres=10, mmin=1)
    assert _groups(r) == {frozenset({0, 4}), frozenset({1, 2}), frozenset({3})}
    lab = {frozenset(r.members(h).tolist()): int(r.halo_id[h]) for h in range(r.nhalo)}
    assert lab[frozenset({0, 4})] == 1
    assert lab[frozenset({1, 2})] == 3  # the lowest index member has ID 2
    assert lab[frozenset({3})] == 4
    assert list(r.halo_id) == [1, 3, 4]  # ascending labels


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_bridge_across_each_face(axis):
    a = [0.5, 0.5, 0.5]
    b = [0.5, 0.5, 0.5]
    a[axis] = 0.004
    b[axis] = 0.994  # periodic distance 0.01 < 0.02
    pos = _box([a, [0.3, 0.3, 0.3], b])
    r = O.fof(pos, np.array([5, 6, 4]), percolation=0.2, nres=10, mmin=2)
    assert r.nbridges == 1
    assert r.nhalo == 1 and r.halo_mass[0] == 2
    # merged to the smaller of the two scan labels
    assert r.halo_id[0] == 4
    assert sorted(r.members(0).tolist()) == [0, 2]
    # centre of mass: the unwrapped mean, wrapped into [0, 1]
    c = r.halo_com[0][axis]
    assert min(abs(c - 0.999), abs(c - (0.999 - 1.0)), abs(c - 1.999)) < 1e-6


def test_bridge_across_a_corner():
    pos = _box([[0.003, 0.003, 0.5], [0.995, 0.996, 0.5]])
    r = O.fof(pos, np.array([1, 2]), percolation=0.2, nres=10, mmin=2)
    assert r.nhalo == 1 and r.halo_mass[0] == 2


def test_mmin_and_heap_order():
    rng = np.random.default_rng(5)
    centre = np.array([0.5, 0.5, 0.5])
    pos = (centre + rng.normal(0, 0.003, (40, 3))).astype(np.float32)
    far = rng.random((25, 3)).astype(np.float32) * 0.2 + 0.05
    pos = np.concatenate([far[:10], pos, far[10:]]).astype(np.float32)
    ids = rng.permutation(len(pos)) + 100
    r = O.fof(pos, ids, percolation=0.2, nres=10, mmin=20)
    assert r.nhalo >= 1
    big = [h for h in range(r.nhalo) if set(range(10, 50)) <= set(r.members(h).tolist())]
    assert len(big) == 1
    assert all(m >= 20 for m in r.halo_mass)
    assert np.all(np.diff(r.halo_id) > 0)
    # heap order: a restatement of the reference's heapsort on the labels
    lab = r.structure.copy()
    idx = np.arange(len(pos))
    n = len(lab)

    def sift(size, i):
        while True:
            l, rr = 2 * i, 2 * i + 1
            m = l if l <= size and lab[l - 1] > lab[i - 1] else i
            if rr <= size and lab[rr - 1] > lab[m - 1]:
                m = rr
            if m == i:
                return
            lab[[i - 1, m - 1]] = lab[[m - 1, i - 1]]
            idx[[i - 1, m - 1]] = idx[[m - 1, i - 1]]
            i = m

    for i in range(n // 2, 0, -1):
        sift(n, i)
    size = n
    for i in range(n, 1, -1):
        lab[[0, i - 1]] = lab[[i - 1, 0]]
        idx[[0, i - 1]] = idx[[i - 1, 0]]
        size -= 1
        sift(size, 1)
    h = big[0]
    lo = int(np.searchsorted(lab, r.halo_id[h]))
    assert np.array_equal(idx[lo: lo + r.halo_mass[h]], r.members(h))


def test_observables_known_answer():
    pos = _box([[0.2, 0.3, 0.4], [0.21, 0.3, 0.4], [0.2, 0.31, 0.4]])
    vel = np.array([[1, 2, 3], [3, 2, 1], [2, 2, 2]], np.float32)
    r = O.fof(pos, np.array([1, 2, 3]), vel=vel, percolation=0.2, nres=10, mmin=3)
    assert r.nhalo == 1
    x = pos.astype(np.float64)
    com = x.mean(axis=0)
    assert np.allclose(r.halo_com[0], com, atol=1e-15)
    assert np.allclose(r.halo_vel[0], [2, 2, 2], atol=1e-15)
    assert r.halo_radius[0] == pytest.approx(np.sqrt(((x - com) ** 2).sum(1)).max(), rel=1e-15)


def test_refuses_long_linking_length():
    r = O.fof(_box([[0.1, 0.1, 0.1]]), np.array([1]), percolation=0.5, nres=4, mmin=1)
    assert r.status == 5


@pytest.mark.parametrize("nres,seed", [(24, 1), (32, 2), (40, 3)])
def test_partition_matches_independent_periodic_fof(nres, seed):
    pytest.importorskip("scipy")
    rng = np.random.default_rng(seed)
    n = nres ** 3
    pos = rng.random((n, 3), dtype=np.float32)
    k = n // 3
    centres = rng.random((25, 3))
    which = rng.integers(0, 25, k)
    pos[:k] = ((centres[which] + rng.normal(0, 0.6 / nres, (k, 3))) % 1.0).astype(np.float32)
    pos[pos >= 1.0] = 0.0
    ids = rng.permutation(n).astype(np.int64) + 1
    r = O.fof(pos, ids, percolation=0.2, nres=nres, mmin=1)
    assert r.status == 0
    assert _groups(r) == _brute_groups(pos, 0.2 / nres)
    assert r.nbridges > 0
