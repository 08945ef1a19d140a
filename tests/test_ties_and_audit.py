"""Exact ties and near-ties: where the reference's arithmetic (FP64 sums in
file order, quicksort tie orders, main:2477-2571) and the canonical
arithmetic of the GPU (int64 fixed point, ties to the lower input index)
can part ways, and what that changes in the outputs.

The crossing loop (main:2040-2100) cannot stop inside a group of equal
distances once it is past its ten forced steps: if the (i-1)-th and i-th
sorted distances are equal, the overdensity at i is i/V(r) > (i-1)/V(r),
which was above delta.  So N_delta, R_delta and the member SET of every
halo with N_delta >= 10 (every kept halo, since Mmin >= 10) do not depend
on the sort's tie order; only the order of members at equal distance does.
The one place a tie can sit at the cut is a stop at the tenth step
(N_delta = 9, always rejected, but its nine particles are still claimed).
These tests build boxes with thousands of exact ties (exact-lattice balls)
and check exactly that, and they count on the configuration-1 box (128^3)
every step where the two arithmetics could disagree.
"""

import numpy as np
import pytest

from tests.boxes import tie_ball_box

TIE_CENTRES = [(15.5, 15.5, 15.5), (31.5, 15.5, 15.5)]  # 16 cells apart: independent seeds


def _members(r, h):
    return r.member_index[r.member_offset[h] : r.member_offset[h + 1]]


@pytest.mark.parametrize("delta", [1000.0, 200.0])
def test_distance_ties_leave_the_member_set_unchanged(oracle, delta):
    pos, ids, balls = tie_ball_box(32, TIE_CENTRES)
    p = oracle.Params(nx=32, delta=delta, nmin=10)
    rr = oracle.run(p, pos, ids, oracle.REFERENCE)
    rc = oracle.run(p, pos, ids, oracle.CANONICAL)
    assert rr.status == rc.status == 0 and rr.nhalo == rc.nhalo == 2
    a = oracle.arithmetic_audit(p, pos, ids)
    assert a["dist_tie_members"] > 0  # the members hold exact ties
    # a tie at the cut only ever follows a forced tenth step (rejected halo)
    assert a["dist_tie_cut"] == 0 or a["dist_tie_cut_nmax"] < 10
    assert np.array_equal(rr.halo_mass, rc.halo_mass)
    assert np.array_equal(rr.halo_id, rc.halo_id)
    assert np.array_equal(rr.halo_rdelta, rc.halo_rdelta)
    assert np.array_equal(rr.halo_profile, rc.halo_profile)
    assert np.array_equal(rr.halo_mass2, rc.halo_mass2)
    if delta == 1000.0:
        # the stop lies inside the ball's shell lattice, at a shell boundary
        assert 10 < rr.halo_mass[0] < balls[0].size
    order_differs = False
    for h in range(rr.nhalo):
        mr, mc = _members(rr, h), _members(rc, h)
        assert np.array_equal(np.sort(mr), np.sort(mc))
        order_differs |= not np.array_equal(mr, mc)
        # members are in ascending distance in both; they differ only inside
        # groups of equal distance
        c = rc.halo_cidx[h]
        pg = (pos.astype(np.float64) * 32).astype(np.float32).astype(np.float64)
        d2r = ((pg[mr] - pg[c]) ** 2).sum(1)
        d2c = ((pg[mc] - pg[c]) ** 2).sum(1)
        assert np.all(np.diff(d2r) >= 0) and np.array_equal(d2r, d2c)
    assert order_differs  # the quicksort tie order is really in effect


def test_exact_density_ties_between_independent_balls(oracle):
    """Two identical balls listed in the same order: their particles have
    exactly equal rho in both arithmetics, so the seed list is full of exact
    ties that quicksort and the index rule order differently.  The seeds of
    the two balls do not depend on each other, so the halos come out the
    same; the seed order (and with it halo_rank) differs only inside groups
    of equal rho."""
    pos, ids, balls = tie_ball_box(32, TIE_CENTRES)
    p = oracle.Params(nx=32, nmin=10)
    a = oracle.arithmetic_audit(p, pos, ids)
    assert a["rho_differ"] == 0
    assert a["seed_exact_ties"] > 100 and a["seed_order_moved"] > 0
    assert a["halos_one_run_only"] == a["halos_mass_differ"] == a["halos_members_differ"] == 0
    r_ref = oracle.rho(p, pos, oracle.REFERENCE)
    s_ref, n_ref = oracle.tri_cic(r_ref, oracle.REFERENCE)
    s_can, n_can = oracle.tri_cic(r_ref, oracle.CANONICAL)
    assert n_ref == n_can
    # same multiset of keys at every rank: the orders differ only among ties
    assert np.array_equal(1.0 / r_ref[s_ref[:n_ref]], 1.0 / r_ref[s_can[:n_can]])


@pytest.mark.slow
def test_configuration_1_box_has_no_arithmetic_divergence(oracle):
    """The 128^3 configuration-1 box (halo N in [20, 2e4], -nx 128 -min 100
    -del 200): every step where the reference's arithmetic and the canonical
    one could decide differently, counted.  None does: the GPU's canonical
    results are the reference's results on this workload."""
    from psod_b200 import synth

    b = synth.make_box(128, nmax_halo=20000, seed=20261203)
    a = oracle.arithmetic_audit(oracle.Params(nx=128), b.pos.numpy(), b.ids.numpy())
    print(a)
    assert a["status"] == (0, 0) and a["nhalo"][0] == a["nhalo"][1] > 900
    assert 0 < a["rho_max_rel"] < 1e-11  # fixed point at 2^-40 against FP64 sums
    assert a["seed_order_moved"] == 0 and a["seed_exact_ties"] == 0
    assert a["refine_seeds"] > 2000 and a["refine_flips"] == 0
    assert a["dist_tie_cut"] == 0
    assert a["halos_one_run_only"] == a["halos_mass_differ"] == a["halos_rdelta_differ"] == 0
    assert a["halos_members_differ"] == 0
