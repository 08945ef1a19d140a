"""Scheduling thresholds (psod_set_tuning) and their autotuner
(psod_autotune): every setting gives the same halo table, bit for bit,
because each threshold only chooses which kernel or pass does a piece of
work."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from psod_b200 import synth  # noqa: E402
from psod_b200.sod import PsodError, SphericalOverdensity  # noqa: E402

FIELDS = ("halo_id", "halo_mass", "halo_rank", "halo_center", "halo_rdelta", "halo_mass2", "halo_mextra",
          "halo_profile", "member_offset", "member_index")


def same(a, b):
    return all(np.array_equal(getattr(a, f), getattr(b, f)) for f in FIELDS)


def test_thresholds_do_not_change_the_table():
    box = synth.make_box(64, seed=12, nmax_halo=8000)
    s = SphericalOverdensity(64, mode=1, delta_extra=(500.0,))
    s.load(box.pos, box.ids)
    assert s.get_tuning() == dict(warp_cross_min_ready=2048, bound_min_cand=4096, tail_max_ready=256,
                                  tail_max_cand=1024)
    s.run()
    ref = s.halos()
    for t in (dict(warp_cross_min_ready=1, bound_min_cand=256, tail_max_ready=0, tail_max_cand=256),
              dict(warp_cross_min_ready=1 << 30, bound_min_cand=8192, tail_max_ready=100000, tail_max_cand=8192)):
        s.set_tuning(**t)
        s.spherover()
        assert same(s.halos(), ref), t
    with pytest.raises(PsodError):
        s.set_tuning(bound_min_cand=100)
    with pytest.raises(PsodError):
        s.set_tuning(tail_max_cand=9000, bound_min_cand=4096)
    r = s.autotune()
    assert r["runs"] >= 10 and r["ms_best"] > 0
    assert same(s.halos(), ref)
    s.close()
