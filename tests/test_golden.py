"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py).

CPU: the fixtures' closed-form answers hold, and the oracle reproduces every
stored output.  GPU: the sm_100a path through the C-ABI reproduces the
canonical outputs bit for bit, rho within 1e-6 of the reference arithmetic
and the reference's N_delta, IDs, R_delta and member sets.
"""

import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ("lattice16", "ball24", "cluster32")
RHO_RTOL = 1e-6


def load(name):
    return dict(np.load(os.path.join(HERE, name + ".npz")))


def params_of(oracle, d):
    return oracle.Params(nx=int(d["nx"]), nbins=int(d["nbins"]), delta_extra=tuple(float(x) for x in d["delta_extra"]))


def test_closed_form_answers():
    d = load("lattice16")
    assert np.all(d["c_rho"] == 8.0) and np.all(d["r_rho"] == 8.0)
    assert int(d["c_npart_new"]) == 1 and d["c_halo_mass"].size == 0
    d = load("ball24")
    assert d["c_halo_mass"].tolist() == [d["ball"].size]
    members = np.sort(d["c_member_index"][d["c_member_offset"][0] : d["c_member_offset"][1]])
    assert np.array_equal(members, d["ball"])
    d = load("cluster32")
    assert d["c_halo_mass"].size >= 10 and d["c_halo_mextra"].shape[1] == 2


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(oracle, name):
    d = load(name)
    p = params_of(oracle, d)
    for mode, pre in ((oracle.CANONICAL, "c_"), (oracle.REFERENCE, "r_")):
        rho = oracle.rho(p, d["pos"], mode)
        assert np.array_equal(rho.astype(d[pre + "rho"].dtype), d[pre + "rho"])
        r = oracle.run(p, d["pos"], d["ids"], mode)
        assert r.status == 0 and r.npart_new == int(d[pre + "npart_new"])
        for k in ("halo_id", "halo_mass", "halo_rank", "halo_center", "halo_rdelta", "halo_mass2", "halo_mextra",
                  "halo_profile", "member_offset", "member_index"):
            assert np.array_equal(getattr(r, k), d[pre + k]), (name, pre, k)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_fixture(name, mode):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from psod_b200.sod import SphericalOverdensity

    d = load(name)
    s = SphericalOverdensity(int(d["nx"]), mode=mode, nbins=int(d["nbins"]),
                             delta_extra=tuple(float(x) for x in d["delta_extra"]))
    try:
        s.load(d["pos"], d["ids"])
        s.cic()
        rho = s.cicm1()
        isort, npart_new = s.tri_cic()
        s.spherover()
        t = s.halos()
        if mode == 1:
            # caller-supplied buffers: pinned host and device tensors
            from psod_b200.sod import HaloTable

            tdt = {np.dtype(np.int64): torch.int64, np.dtype(np.float32): torch.float32,
                   np.dtype(np.float64): torch.float64}
            for kw in (dict(pin_memory=True), dict(device="cuda")):
                out = HaloTable(**{f: torch.full((getattr(t, f).size + 3,), -7, dtype=tdt[getattr(t, f).dtype], **kw)
                                   for f in HaloTable.__dataclass_fields__})
                u = s.halos(out=out)
                for f in HaloTable.__dataclass_fields__:
                    assert np.array_equal(getattr(u, f).cpu().numpy(), getattr(t, f)), f
    finally:
        s.close()
    # canonical arithmetic: bit-exact
    assert np.array_equal(rho, d["c_rho"])
    assert npart_new == int(d["c_npart_new"]) and np.array_equal(isort, d["c_isort"])
    for k in ("halo_id", "halo_mass", "halo_rank", "halo_center", "halo_rdelta", "halo_mass2", "halo_profile",
              "member_offset", "member_index"):
        assert np.array_equal(np.asarray(getattr(t, k)), d["c_" + k]), k
    if d["delta_extra"].size:
        assert np.array_equal(np.asarray(t.halo_mextra), d["c_halo_mextra"])
    # reference arithmetic: rho within tolerance, halos and member sets equal
    assert np.allclose(rho, d["r_rho"].astype(np.float64), rtol=RHO_RTOL, atol=0.0)
    assert np.array_equal(np.asarray(t.halo_mass), d["r_halo_mass"])
    assert np.array_equal(np.asarray(t.halo_id), d["r_halo_id"])
    assert np.array_equal(np.asarray(t.halo_rdelta), d["r_halo_rdelta"])
    off = d["r_member_offset"]
    for h in range(d["r_halo_mass"].size):
        a = np.sort(np.asarray(t.member_index)[off[h] : off[h + 1]])
        b = np.sort(d["r_member_index"][off[h] : off[h + 1]])
        assert np.array_equal(a, b)
