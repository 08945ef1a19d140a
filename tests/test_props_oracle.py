"""The halo-properties oracle (oracle/psod_oracle_props.c, haloanalyzer's
halo_properties) against answers known in closed form: a two-particle
halo's potential energy and most bound member, a halo across the periodic
boundary, the inertia tensor of a triaxial cloud, the virial quantities
from the particle count, the profile bins' particle counts, and the
sampled potential of a large halo against the exact one."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

MPC = 3.08568e24
MSUN = 1.98892e33
UNITS = dict(unit_l=MPC * 100 / 0.7, unit_d=2.7e-30, unit_t=4.4e17, aexp=1.0, h0=70.0, hz=1.0, delta_vir=178.0,
             levelmin=7)
PI = float(np.float32(3.14159265359879))
G = float(np.float32(6.6731e-08))


def props(pos, vel=None, halos=None, **kw):
    pos = np.asarray(pos, np.float32).reshape(-1, 3)
    if halos is None:
        halos = [np.arange(len(pos))]
    off = np.concatenate([[0], np.cumsum([len(h) for h in halos])])
    mem = np.concatenate(halos)
    args = dict(UNITS)
    args.update(kw)
    return O.halo_properties(off, mem, pos, vel, **args)


def test_virial_quantities_from_the_count():
    pos = np.full((50, 3), 0.5, np.float32) + np.arange(50, dtype=np.float32)[:, None] * 1e-5
    out = props(pos)
    mp = 1.0 / float(2 ** 7) ** 3
    m_vir = 50 * mp * UNITS["unit_d"] * UNITS["unit_l"] ** 3
    r_vir = (3 * m_vir / (4 * PI * 178.0 * UNITS["unit_d"])) ** float(np.float32(1.0) / np.float32(3.0))
    assert out["npart"][0] == 50
    assert out["mvir"][0] == pytest.approx(m_vir / MSUN * 70 / 100, rel=1e-12)
    assert out["rvir"][0] == pytest.approx(r_vir / (MPC / 1e3) * 70 / 100, rel=1e-12)
    assert out["vvir"][0] == pytest.approx(np.sqrt(G * m_vir / r_vir) / 1e5, rel=1e-12)


def test_two_particle_potential_and_most_bound():
    pos = np.array([[0.5, 0.5, 0.5], [0.5 + 1e-4, 0.5, 0.5]], np.float32)
    out = props(pos)
    mp = 1.0 / float(2 ** 7) ** 3
    dx = float(np.float32(0.5 + 1e-4) - np.float32(0.5))
    delta_x = (1.0 / 2 ** 7) / 64
    term = mp * mp / np.sqrt(dx * dx + delta_x ** 2)
    epot = -0.5 * G * (2 * term) * (UNITS["unit_d"] * UNITS["unit_l"] ** 3) ** 2 / UNITS["unit_l"]
    m_vir = 2 * mp * UNITS["unit_d"] * UNITS["unit_l"] ** 3
    r_vir = (3 * m_vir / (4 * PI * 178.0 * UNITS["unit_d"])) ** float(np.float32(1.0) / np.float32(3.0))
    v_vir = np.sqrt(G * m_vir / r_vir)
    norm = 0.5 * m_vir / MSUN * (v_vir / 1e5) ** 2
    assert out["epot"][0] == pytest.approx(epot / (MSUN * 1e10) / norm, rel=1e-6)
    # equal potential sums: the first particle is the most bound (strict >)
    conv = 70 / 100 / 1.0
    assert np.allclose(out["center_pot"][0], pos[0] * UNITS["unit_l"] / MPC * conv, rtol=1e-6)


def test_halo_across_the_boundary():
    rng = np.random.default_rng(3)
    pts = (np.array([0.9995, 0.3, 0.6]) + rng.normal(0, 4e-4, (300, 3))) % 1.0
    out = props(pts.astype(np.float32))
    com = out["com"][0] / (UNITS["unit_l"] / MPC * 0.7)
    # the centre lies at the cluster, near x = 0 or x = 1 of the box
    assert min(abs(com[0] - 0.9995), abs(com[0] + 0.0005), abs(com[0] - 1.9995)) < 2e-4
    assert abs(com[1] - 0.3) < 2e-4 and abs(com[2] - 0.6) < 2e-4
    assert out["rmax"][0] < 5.0  # in R_vir; a particle left a box away would give ~100


def test_inertia_of_a_triaxial_cloud():
    rng = np.random.default_rng(4)
    q = rng.normal(size=(20000, 3)) * np.array([1.0, 0.7, 0.4]) * 1e-3
    out = props((0.5 + q).astype(np.float32))
    a, b, c = out["eig_val"][0]
    assert a > b > c
    assert b / a == pytest.approx(0.7, rel=0.03) and c / a == pytest.approx(0.4, rel=0.03)
    assert abs(abs(out["eig_vec"][0][2]) - 1.0) < 0.01  # the minor axis is z


def test_profile_counts_add_up():
    rng = np.random.default_rng(5)
    pts = 0.5 + rng.normal(0, 2e-3, (5000, 3))
    out = props(pts.astype(np.float32), center_on_mass=True)
    # integrated density at the last bin holds every particle inside it
    mp = 1.0 / float(2 ** 7) ** 3
    r_last = np.exp(100 * 0.1) * (MPC / 1e3)
    m_all = 5000 * mp * UNITS["unit_d"] * UNITS["unit_l"] ** 3
    di = m_all / (float(np.float32(4.0) / np.float32(3.0)) * PI * r_last ** 3) / UNITS["unit_d"]
    assert out["dens_int"][0][-1] == pytest.approx(di, rel=1e-6)
    assert np.all(out["dens"][0] >= 0)


def test_sampled_potential_tracks_the_exact_one():
    rng = np.random.default_rng(6)
    pts = (0.5 + rng.normal(0, 1e-3, (3000, 3))).astype(np.float32)
    exact = props(pts)
    sampled = props(pts, epot_threshold=1000)  # 100 sampled members
    assert sampled["epot"][0] == pytest.approx(exact["epot"][0], rel=0.1)
    assert exact["ekin"][0] == sampled["ekin"][0]
