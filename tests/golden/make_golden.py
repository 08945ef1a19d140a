"""Golden fixtures for the SOD parity tests.

The reference ships no test vectors for this path and cannot be built here
(Fortran + MPI + HDF5), so these fixtures come from the CPU oracle
(oracle/psod_oracle.c, which restates the reference line by line) on three
small boxes.  Two of them have answers known in closed form, which pins the
oracle itself; the third freezes the oracle's output on a clustered box.

  lattice16  cell-centred 16^3 lattice: rho == 8 for every particle, the seed
             list holds only the first particle at rho <= 100, no halo.
  ball24     24^3 lattice with a spherical hole refilled by a compact ball
             (tests/boxes.hole_ball_box): N_200 == ball count, the members
             are the ball.
  cluster32  seeded NFW-mixture 32^3 box (psod_b200.synth.make_box),
             Delta = 200 with extra thresholds 500 and 178 and 48 bins:
             canonical outputs (the GPU's bit-exact target) and reference
             outputs.  The reference-arithmetic rho is stored as float32
             (it is only compared within 1e-6 relative).

Each .npz holds the inputs (positions, IDs, parameters) and the expected
outputs.  Run from the repository root:

    python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from tests.boxes import hole_ball_box, lattice_box  # noqa: E402

HALO_KEYS = ("halo_id", "halo_mass", "halo_rank", "halo_center", "halo_rdelta", "halo_mass2", "halo_mextra",
             "halo_profile", "member_offset", "member_index")


def outputs(params: O.Params, pos, ids, mode, prefix: str) -> dict:
    rho = O.rho(params, pos, mode)
    isort, npart_new = O.tri_cic(rho, mode)
    r = O.run(params, pos, ids, mode)
    assert r.status == 0, r.status
    out = {f"{prefix}rho": rho, f"{prefix}isort": isort[:npart_new], f"{prefix}npart_new": np.int64(npart_new)}
    for k in HALO_KEYS:
        out[prefix + k] = getattr(r, k)
    return out


def save(name: str, params: O.Params, pos, ids, modes, extra=None, f32_keys=()):
    d = {
        "pos": np.ascontiguousarray(pos, np.float32),
        "ids": np.ascontiguousarray(ids, np.int64),
        "nx": np.int64(params.nx),
        "nbins": np.int64(params.nbins),
        "delta_extra": np.asarray(params.delta_extra, np.float64),
    }
    for mode, prefix in modes:
        d.update(outputs(params, pos, ids, mode, prefix))
    if extra:
        d.update(extra)
    for k in f32_keys:
        d[k] = d[k].astype(np.float32)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **d)
    print(f"{path}: {d['pos'].shape[0]} particles, {os.path.getsize(path)} bytes")


def main():
    O.build()
    # lattice: rho == 8 exactly, one seed, no halo
    pos, ids = lattice_box(16)
    p = O.Params(nx=16)
    save("lattice16", p, pos, ids, [(O.CANONICAL, "c_"), (O.REFERENCE, "r_")])

    # isolated ball: N_200 == ball count
    pos, ids, balls = hole_ball_box(24, [(11.3, 12.6, 9.9)], r_hole=3.6, r_ball=0.3)
    p = O.Params(nx=24)
    save("ball24", p, pos, ids, [(O.CANONICAL, "c_"), (O.REFERENCE, "r_")], {"ball": balls[0]})

    # clustered box with three thresholds and 48 bins
    from psod_b200 import synth

    b = synth.make_box(32, nmax_halo=3000, seed=20261203)
    pos = np.ascontiguousarray(b.pos.cpu().numpy() if hasattr(b.pos, "cpu") else b.pos, np.float32)
    ids = np.ascontiguousarray(b.ids.cpu().numpy() if hasattr(b.ids, "cpu") else b.ids, np.int64)
    p = O.Params(nx=32, nbins=48, delta_extra=(500.0, 178.0))
    save("cluster32", p, pos, ids, [(O.CANONICAL, "c_"), (O.REFERENCE, "r_")], f32_keys=("r_rho",))


if __name__ == "__main__":
    main()
