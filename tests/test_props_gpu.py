"""GPU halo properties (psod_halo_properties through the C-ABI) against the
oracle's restatement of haloanalyzer's halo_properties
(oracle/psod_oracle_props.c), on the SOD table and on the FoF catalogue of
clustered boxes, members in the tables' order.

Each member's potential sum is formed in the same order on both sides, so
the most bound member and the profiles' bin counts are identical; the other
sums run in another order on the GPU, so real(4) outputs may differ by an
ulp (rtol 1e-6) and real(8) ones by rounding (rtol 1e-12)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from psod_b200 import synth  # noqa: E402
from psod_b200.sod import PsodError, SphericalOverdensity  # noqa: E402

MPC = 3.08568e24
UNITS = dict(unit_l=MPC * 100 / 0.7, unit_d=2.7e-30, unit_t=4.4e17, aexp=1.0, h0=70.0, hz=1.0, delta_vir=178.0,
             levelmin=6)
F32_RTOL = 1e-6
F64_RTOL = 1e-12


def compare(g, o, nh):
    assert np.array_equal(g["npart"], o["npart"])
    for f in ("mvir", "rvir", "rvircom", "vvir"):
        assert np.allclose(g[f], o[f], rtol=F64_RTOL, atol=0), f
    assert np.array_equal(g["center_pot"], o["center_pot"])  # same most bound member
    for f in ("com", "comv", "rmax", "vmax", "dispx", "dispv", "ekin", "epot", "lambda", "lambda_prime", "eig_val",
              "circ", "delta_vals", "dens", "dens_int", "vcirc", "dens178", "dens_int178"):
        a, b = g[f], o[f]
        ok = np.isclose(a, b, rtol=F32_RTOL, atol=1e-30) | (np.isnan(a) & np.isnan(b))
        assert ok.all(), (f, np.argwhere(~ok)[:3], a[~ok][:3], b[~ok][:3])
    # the minor axis up to its sign
    s = np.sign(np.sum(g["eig_vec"] * o["eig_vec"], axis=1))[:, None]
    assert np.allclose(g["eig_vec"], s * o["eig_vec"], rtol=1e-5, atol=1e-6)
    assert np.allclose(np.abs(g["cos_alpha"]), np.abs(o["cos_alpha"]), rtol=1e-9, atol=1e-12, equal_nan=True)


@pytest.mark.parametrize("source,threshold", [("sod", 30000), ("fof", 30000), ("sod", 300)])
def test_properties_match_oracle(oracle, source, threshold):
    nx = 48
    box = synth.make_box(nx, seed=91, nmax_halo=6000)
    pos = box.pos.numpy()
    vel = np.random.default_rng(9).normal(0, 0.3, pos.shape).astype(np.float32)
    s = SphericalOverdensity(nx, nmin=20)
    s.load(box.pos, box.ids, vel=torch.from_numpy(vel))
    if source == "sod":
        s.run()
        t = s.halos()
        off, mem = t.member_offset, t.member_index
    else:
        s.fof(percolation=0.2, mmin=20)
        t = s.fof_halos()
        off, mem = t.member_offset, t.member_index
    g, st = s.halo_properties(**UNITS, source=source, epot_threshold=threshold)
    s.close()
    nh = len(off) - 1
    assert nh > 20 and st["nhalo"] == nh
    o = oracle.halo_properties(off, mem, pos, vel, **UNITS, epot_threshold=threshold)
    compare(g, o, nh)


def test_properties_need_a_table():
    box = synth.make_box(16, seed=3, nmax_halo=500)
    s = SphericalOverdensity(16)
    s.load(box.pos, box.ids)
    with pytest.raises(PsodError):
        s.halo_properties(**UNITS, source="sod")
    with pytest.raises(PsodError):
        s.halo_properties(**UNITS, source="fof")
    s.close()
