"""Known-answer particle boxes for the SOD tests.

hole_ball_box: a cell-centred lattice with the lattice points inside a
sphere of radius ``r_hole`` cells removed and the same number of particles
packed into a ball of radius ``r_ball`` at the sphere's centre.  With
``r_hole - r_ball`` well above the ball's R_200, the reference's crossing
loop (main:2040-2100) stops at the first lattice particle, so N_200 equals
the ball's particle count exactly and the members are exactly the ball.
"""

from __future__ import annotations

import numpy as np


def lattice_points(nx: int) -> np.ndarray:
    g = np.arange(nx, dtype=np.float64)
    zz, yy, xx = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([xx, yy, zz], -1).reshape(-1, 3) + 0.5  # grid units


def _wrap_f32(p_grid: np.ndarray, nx: int) -> np.ndarray:
    x = np.mod(p_grid / nx, 1.0)
    xf = x.astype(np.float32)
    xf[xf >= 1.0] = 0.0
    return xf


def hole_ball_box(nx: int, centres, r_hole: float, r_ball: float, seed: int = 3, squeeze=None):
    """Returns (pos float32 (N,3) box units, ids int64, ball index lists).

    ``centres`` in grid units; one ball per centre.  ``squeeze`` optionally
    gives, per ball, an exponent > 1/3 that concentrates the ball radially.
    """
    rng = np.random.default_rng(seed)
    lat = lattice_points(nx)
    keep = np.ones(lat.shape[0], bool)
    balls = []
    counts = []
    for c in centres:
        c = np.asarray(c, np.float64)
        d = lat - c
        d -= nx * np.round(d / nx)
        inside = (d * d).sum(1) <= r_hole * r_hole
        inside &= keep
        counts.append(int(inside.sum()))
        keep &= ~inside
    pts = [lat[keep]]
    for bi, (c, k) in enumerate(zip(centres, counts)):
        u = rng.random(k)
        expo = 1.0 / 3.0 if squeeze is None else squeeze[bi]
        r = r_ball * u**expo
        v = rng.normal(size=(k, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        pts.append(np.asarray(c, np.float64) + r[:, None] * v)
    allp = np.concatenate(pts, 0)
    pos = _wrap_f32(allp, nx)
    n = pos.shape[0]
    perm = rng.permutation(n)
    pos = pos[perm]
    ids = rng.permutation(n).astype(np.int64) + 1000
    # index lists of each ball in the shuffled order
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    start = int(keep.sum())
    for k in counts:
        balls.append(np.sort(inv[start : start + k]))
        start += k
    return np.ascontiguousarray(pos), ids, balls


def holes_and_balls(nx: int, holes, balls, seed: int = 3):
    """Lattice minus spherical holes [(centre, r_hole)], refilled with balls
    [(centre, r_ball, count)]; the last ball takes whatever count is left so
    the total stays nx**3.  Returns (pos, ids, ball index lists)."""
    rng = np.random.default_rng(seed)
    lat = lattice_points(nx)
    keep = np.ones(lat.shape[0], bool)
    for c, rh in holes:
        d = lat - np.asarray(c, np.float64)
        d -= nx * np.round(d / nx)
        keep &= (d * d).sum(1) > rh * rh
    free = int((~keep).sum())
    counts = [b[2] for b in balls[:-1]]
    counts.append(free - sum(counts))
    assert counts[-1] > 0
    pts = [lat[keep]]
    for (c, rb, _), k in zip(balls, counts):
        r = rb * rng.random(k) ** (1.0 / 3.0)
        v = rng.normal(size=(k, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        pts.append(np.asarray(c, np.float64) + r[:, None] * v)
    pos = _wrap_f32(np.concatenate(pts, 0), nx)
    n = pos.shape[0]
    perm = rng.permutation(n)
    pos = pos[perm]
    ids = rng.permutation(n).astype(np.int64) + 1000
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    out = []
    start = int(keep.sum())
    for k in counts:
        out.append(np.sort(inv[start : start + k]))
        start += k
    return np.ascontiguousarray(pos), ids, out


def lattice_box(nx: int):
    pos = _wrap_f32(lattice_points(nx), nx)
    ids = np.arange(nx**3, dtype=np.int64)
    return pos, ids


def ref_d2(pos_box: np.ndarray, nx: int, centre_idx: int) -> np.ndarray:
    """The reference's FP64 minimum-image d2 (main:2014-2020) to a particle."""
    pg = (pos_box.astype(np.float64) * nx).astype(np.float32).astype(np.float64)
    c = pg[centre_idx]
    d = np.abs(pg - c)
    d = np.minimum(d, nx - d)
    return (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]


def shell_ball_points(centre, core_h, core_r, outer_h, outer_r):
    """Points on two nested cubic lattices around ``centre`` (grid units): a
    fine core (spacing ``core_h`` cells, radius ``core_r``) and a coarser
    shell region (spacing ``outer_h``, out to ``outer_r``).  With the centre
    and both spacings powers of two fractions of a cell, every coordinate
    and every squared distance to the centre is exact in float32 / FP64, so
    whole shells of points lie at exactly equal distances."""
    pts = [np.zeros((1, 3))]
    for h, r0, r1 in ((core_h, 0.0, core_r), (outer_h, core_r, outer_r)):
        m = int(np.floor(r1 / h))
        g = np.arange(-m, m + 1, dtype=np.float64) * h
        zz, yy, xx = np.meshgrid(g, g, g, indexing="ij")
        p = np.stack([xx, yy, zz], -1).reshape(-1, 3)
        d2 = (p * p).sum(1)
        pts.append(p[(d2 > r0 * r0) & (d2 <= r1 * r1)])
    return np.asarray(centre, np.float64) + np.unique(np.concatenate(pts), axis=0)


def tie_ball_box(nx: int, centres, r_hole: float = 3.6, core_h=1 / 32, core_r=0.1, outer_h=1 / 8, outer_r=0.45):
    """A cell-centred lattice with holes of radius ``r_hole`` around each
    centre, each hole holding the same exact-lattice ball
    (``shell_ball_points``).  Particles are listed lattice first, then the
    balls one after the other in the same order, so that translated copies
    deposit identical CIC contributions in the same order and their
    particles get exactly equal densities in both arithmetics.  Returns
    (pos float32 box units, ids int64, per-ball index arrays)."""
    lat = lattice_points(nx)
    keep = np.ones(lat.shape[0], bool)
    for c in centres:
        d = lat - np.asarray(c, np.float64)
        d -= nx * np.round(d / nx)
        keep &= (d * d).sum(1) > r_hole * r_hole
    parts = [lat[keep]]
    balls = []
    start = int(keep.sum())
    for c in centres:
        b = shell_ball_points(c, core_h, core_r, outer_h, outer_r)
        parts.append(b)
        balls.append(np.arange(start, start + b.shape[0]))
        start += b.shape[0]
    pos = _wrap_f32(np.concatenate(parts, 0), nx)
    ids = np.arange(pos.shape[0], dtype=np.int64) * 7 + 11
    return pos, ids, balls
