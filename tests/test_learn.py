"""Learned radius bracket: the network's kernels against a numpy restatement,
training on the engine's own samples, and the bracket's effect on a run.

The reference has no learned component; the checks are (a) the numpy
restatement's gradient against finite differences (CPU), (b) the GPU forward
and gradient kernels against the restatement with the same bfloat16 rounding
points, (c) training lowers the loss, (d) the learned mode gives the batched
mode's halo table bit for bit while its crossing search needs fewer ball
passes (the network's first ball is never below the batched mode's, so
every seed needs at most as many passes).
"""

import numpy as np
import pytest

from tests import mlp_ref as R


def _xt(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1.5, (n, R.NF)).astype(np.float32)
    t = rng.normal(0, 1.0, (n, R.NOUT)).astype(np.float32)
    return x, t


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, -2.5, 3.0e-39], np.float32)
    r = R.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0 + 2**-6)  # tie rounds up to the even neighbour
    assert r[3] == -2.5 and r[4] > 0


def test_reference_gradient_matches_finite_differences():
    blob = R.random_blob(3).astype(np.float64)
    x, t = _xt(64, 4)
    g, _ = R.gradient(blob, x, t, emulate=False)
    rng = np.random.default_rng(5)
    real = np.concatenate([
        (R.OW1 + np.arange(R.HID)[:, None] * R.IN + np.arange(R.NF)[None, :]).ravel(),
        np.arange(R.OB1, R.OW3),
        (R.OW3 + np.arange(R.NOUT)[:, None] * R.HID + np.arange(R.HID)[None, :]).ravel(),
        np.arange(R.OB3, R.OB3 + R.NOUT),
    ])
    h = 1e-6
    for k in rng.choice(real, 60, replace=False):
        bp, bm = blob.copy(), blob.copy()
        bp[R.NNORM + k] += h
        bm[R.NNORM + k] -= h
        fd = (R.loss64(bp, x, t) - R.loss64(bm, x, t)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-4 * abs(g[k]), (k, fd, g[k])


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from psod_b200.sod import SphericalOverdensity

    return SphericalOverdensity


def _blocks(g):
    return {"W1": g[R.OW1:R.OB1], "b1": g[R.OB1:R.OW2], "W2": g[R.OW2:R.OB2], "b2": g[R.OB2:R.OW3],
            "W3": g[R.OW3:R.OB3], "b3": g[R.OB3:R.NPARAM]}


@pytest.mark.gpu
def test_gpu_forward_and_gradient_match_reference():
    SO = _gpu()
    blob = R.random_blob(11)
    x, t = _xt(1000, 12)  # not a multiple of the 64-row tile
    with SO(32, mode=2) as s:
        s.learn_set_model(blob)
        assert np.array_equal(s.learn_get_model(), blob)
        y = s.learn_forward(x)
        g, loss = s.learn_gradient(x, t)
    ye = R.forward(blob, x, emulate=True)
    assert np.allclose(y, ye, rtol=2e-3, atol=5e-3), np.abs(y - ye).max()
    ge, le = R.gradient(blob, x, t, emulate=True)
    g64, l64 = R.gradient(blob, x, t, emulate=False)
    assert abs(loss - le) <= 1e-3 * le
    for name, a in _blocks(g).items():
        e = _blocks(ge)[name]
        f = _blocks(g64)[name]
        assert np.linalg.norm(a - e) <= 1e-2 * np.linalg.norm(e) + 1e-7, name
        assert np.linalg.norm(a - f) <= 6e-2 * np.linalg.norm(f) + 1e-6, name
    # padding stays zero
    assert np.all(g[R.OW1:R.OB1].reshape(R.HID, R.IN)[:, R.NF:] == 0)
    assert np.all(g[R.OW3:R.OB3].reshape(R.OUTP, R.HID)[R.NOUT:] == 0)


@pytest.mark.gpu
def test_learned_bracket_trains_and_keeps_results():
    SO = _gpu()
    from psod_b200 import synth

    box = synth.make_box(128, nmax_halo=20000, seed=7, device="cuda")
    # samples from the batched run
    with SO(128, mode=1) as s:
        s.learn_collect(1 << 20)
        s.load(box.pos, box.ids)
        st_b = s.run()
        tb = s.halos()
        x, t = s.learn_samples()
        assert x.shape[0] == st_b["bracket_seeds"] > 500
        assert np.all(np.isfinite(x)) and np.all(np.isfinite(t))
        loss = s.learn_train(epochs=20, batch=256, lr=1e-3, seed=1)
        model = s.learn_get_model()
    assert loss[-1] < 0.5 * loss[0], loss
    # the learned mode: same halo table, fewer records in the crossing balls
    with SO(128, mode=2) as s:
        s.learn_set_model(model)
        s.load(box.pos, box.ids)
        st_l = s.run()
        tl = s.halos()
    for f in ("halo_id", "halo_mass", "halo_rank", "halo_center", "halo_rdelta", "halo_mass2", "halo_profile",
              "member_offset", "member_index", "member_id"):
        assert np.array_equal(getattr(tl, f), getattr(tb, f)), f
    assert st_l["bracket_seeds"] == st_b["bracket_seeds"]
    hit_b = st_b["bracket_hits"] / st_b["bracket_seeds"]
    hit_l = st_l["bracket_hits"] / st_l["bracket_seeds"]
    print(f"bracket hits: batched {hit_b:.3f}, learned {hit_l:.3f}; records in crossing balls: "
          f"batched {st_b['cross_records']}, learned {st_l['cross_records']}; ball passes: "
          f"batched {st_b['cross_balls']}, learned {st_l['cross_balls']}")
    assert st_l["cross_balls"] < st_b["cross_balls"]
    assert hit_l >= hit_b


@pytest.mark.gpu
def test_learned_bracket_with_fof_features():
    """The configuration the task names: inputs from the seed's FoF group
    (log N_FoF, inertia axis ratios, log peak overdensity, peak - centre of
    mass offset, R_FoF, RMS radius), targets log(R_stop / R_FoF) and the
    centre offset.  Same halo table as the batched mode."""
    SO = _gpu()
    from psod_b200 import synth

    box = synth.make_box(128, nmax_halo=20000, seed=7, device="cuda")
    with SO(128, mode=1) as s:
        s.load(box.pos, box.ids)
        s.fof(percolation=0.2, mmin=20)
        s.fof_release()
        s.learn_set_features("fof")
        s.learn_collect(1 << 20)
        st_b = s.run()
        tb = s.halos()
        x, t = s.learn_samples()
        # samples only for seeds inside FoF halos, with finite features
        assert 100 < x.shape[0] <= st_b["bracket_seeds"]
        assert np.all(np.isfinite(x)) and np.all(np.isfinite(t))
        assert np.all(x[:, 8] > 0) and np.all(x[:, 0] >= np.log(20) - 1e-6)
        assert np.all((x[:, 1:4] > 0) & (x[:, 1:4] <= 1.0 + 1e-6))
        assert np.all(t[:, 1] >= 0)  # centre offsets (cells)
        loss = s.learn_train(epochs=20, batch=256, lr=1e-3, seed=1)
        model = s.learn_get_model()
    assert loss[-1] < loss[0], loss
    with SO(128, mode=2) as s:
        s.learn_set_features("fof")
        s.learn_set_model(model)
        s.load(box.pos, box.ids)
        from psod_b200.sod import PsodError

        with pytest.raises(PsodError):  # no FoF catalogue yet
            s.run()
        s.fof(percolation=0.2, mmin=20)
        st_l = s.run()
        tl = s.halos()
    for f in ("halo_id", "halo_mass", "halo_rank", "halo_center", "halo_rdelta", "halo_mass2", "halo_profile",
              "member_offset", "member_index", "member_id"):
        assert np.array_equal(getattr(tl, f), getattr(tb, f)), f
    print(f"FoF features: bracket hits batched {st_b['bracket_hits'] / st_b['bracket_seeds']:.3f}, "
          f"learned {st_l['bracket_hits'] / max(1, st_l['bracket_seeds']):.3f}; ball passes batched "
          f"{st_b['cross_balls']}, learned {st_l['cross_balls']}")
