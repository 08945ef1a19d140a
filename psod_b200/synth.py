"""Seeded synthetic clustered boxes: the stand-in for the reference's RAMSES
particle cubes, which are not available.

A box of ``nx**3`` equal-mass particles with float32 positions in the
periodic unit cube and shuffled int64 IDs. A fraction ``halo_frac`` (0.45)
of the particles lie in halos: the halo sizes follow ``dN/dN_h ~ N_h**-1.9``
on ``[nmin_halo, nmax_halo]``, each halo has a uniform random centre, and its
particles are drawn from an NFW profile with concentration ``c ~ U[4, 12]``
truncated at ``1.5 * R200``. R200 comes from the halo size at a mean density
of one particle per cell. The remaining particles are uniform. Velocities are
zero: SOD arithmetic never reads them.

Optional heavy clusters (the stress box) add ``n_clusters`` halos of
``cluster_size`` particles with concentration 4 and axis ratios 1:0.8:0.6.

Works on any torch device. A CPU run is fully reproducible from its seed. On
CUDA the random stream differs, but it is reproducible from run to run.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch


@dataclass
class Box:
    pos: torch.Tensor  # (N, 3) float32 in [0, 1)
    ids: torch.Tensor  # (N,) int64
    nx: int
    halo_sizes: torch.Tensor  # (H,) int64, generator halos
    halo_centres: torch.Tensor  # (H, 3) float64

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


def _power_law(gen, n, a, b, alpha, device):
    """Inverse-CDF samples of p(N) ~ N**-alpha on [a, b] (float64)."""
    u = torch.rand(n, generator=gen, dtype=torch.float64, device=device)
    e = 1.0 - alpha
    return (a**e + u * (b**e - a**e)) ** (1.0 / e)


def _nfw_radius(u_mass, xmax, iters=60):
    """Solve m(x) = u * m(xmax) for x in [0, xmax], m(x) = ln(1+x) - x/(1+x).

    Bisection in float64: robust and vectorised.
    """
    target = u_mass * (torch.log1p(xmax) - xmax / (1.0 + xmax))
    lo = torch.zeros_like(target)
    hi = xmax.expand_as(target).clone()
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        m = torch.log1p(mid) - mid / (1.0 + mid)
        below = m < target
        lo = torch.where(below, mid, lo)
        hi = torch.where(below, hi, mid)
    return 0.5 * (lo + hi)


def _unit_vectors(gen, n, device):
    v = torch.randn(n, 3, generator=gen, dtype=torch.float64, device=device)
    return v / v.norm(dim=1, keepdim=True).clamp_min(1e-300)


def _sample_halo_particles(gen, sizes, centres, conc, nx, ntot, axes=None):
    """Particles for halos of given sizes (int64), centres (H,3) and
    concentrations (H,), as float64 box-unit positions (unwrapped)."""
    device = sizes.device
    h = sizes.numel()
    if h == 0:
        return torch.zeros(0, 3, dtype=torch.float64, device=device)
    owner = torch.repeat_interleave(torch.arange(h, device=device), sizes)
    m = owner.numel()
    # R200 in box units: N_h = 200 * mean * (4/3) pi R^3, mean = ntot per unit volume
    r200 = (3.0 * sizes.double() / (4.0 * math.pi * 200.0 * ntot)) ** (1.0 / 3.0)
    c = conc[owner]
    xmax = 1.5 * c  # truncation at 1.5 R200, in units of r_s
    u = torch.rand(m, generator=gen, dtype=torch.float64, device=device)
    x = _nfw_radius(u, xmax)
    r = x / c * r200[owner]
    d = _unit_vectors(gen, m, device)
    if axes is not None:
        d = d * axes.to(device=device, dtype=torch.float64)
    return centres[owner] + r[:, None] * d


def _to_f32_unit(x):
    """Wrap float64 box positions into [0,1) and round to float32 < 1."""
    x = torch.remainder(x, 1.0)
    xf = x.to(torch.float32)
    return torch.where(xf >= 1.0, torch.zeros_like(xf), xf)


def make_box(
    nx: int,
    seed: int = 20261203,
    halo_frac: float = 0.45,
    nmin_halo: int = 20,
    nmax_halo: int = 20000,
    alpha: float = 1.9,
    conc_range=(4.0, 12.0),
    n_clusters: int = 0,
    cluster_size: int = 5_000_000,
    device="cpu",
    shuffle: bool = True,
) -> Box:
    """Generate a clustered periodic box with ``nx**3`` particles."""
    device = torch.device(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    ntot = nx**3
    n_halo_target = int(round(halo_frac * ntot))

    # heavy clusters first (stress box), then the power-law population
    cl_pos = torch.zeros(0, 3, dtype=torch.float64, device=device)
    n_cl = 0
    if n_clusters > 0:
        n_cl = min(n_clusters * cluster_size, n_halo_target)
        per = n_cl // n_clusters
        sizes = torch.full((n_clusters,), per, dtype=torch.int64, device=device)
        n_cl = per * n_clusters
        centres = torch.rand(n_clusters, 3, generator=gen, dtype=torch.float64, device=device)
        conc = torch.full((n_clusters,), 4.0, dtype=torch.float64, device=device)
        axes = torch.tensor([1.0, 0.8, 0.6], dtype=torch.float64)
        cl_pos = _sample_halo_particles(gen, sizes, centres, conc, nx, ntot, axes=axes)

    remaining = n_halo_target - n_cl
    # draw halo sizes in batches until the target is covered
    mean_size = _mean_power_law(nmin_halo, nmax_halo, alpha)
    sizes_list = []
    total = 0
    while total < remaining:
        batch = max(16, int(1.2 * (remaining - total) / mean_size) + 16)
        s = _power_law(gen, batch, float(nmin_halo), float(nmax_halo), alpha, device)
        s = torch.floor(s).to(torch.int64).clamp(nmin_halo, nmax_halo)
        cs = torch.cumsum(s, 0)
        keep = int(torch.searchsorted(cs, torch.tensor(remaining - total, device=device), right=False).item()) + 1
        keep = min(keep, batch)
        s = s[:keep]
        sizes_list.append(s)
        total += int(s.sum().item())
    sizes = torch.cat(sizes_list) if sizes_list else torch.zeros(0, dtype=torch.int64, device=device)
    if total > remaining and sizes.numel() > 0:
        sizes[-1] -= total - remaining
        if sizes[-1] <= 0:
            sizes = sizes[:-1]
    h = sizes.numel()
    centres = torch.rand(h, 3, generator=gen, dtype=torch.float64, device=device)
    conc = conc_range[0] + (conc_range[1] - conc_range[0]) * torch.rand(
        h, generator=gen, dtype=torch.float64, device=device
    )
    hp = _sample_halo_particles(gen, sizes, centres, conc, nx, ntot)

    n_uniform = ntot - hp.shape[0] - cl_pos.shape[0]
    up = torch.rand(n_uniform, 3, generator=gen, dtype=torch.float64, device=device)
    allpos = torch.cat([cl_pos, hp, up], 0)
    pos = _to_f32_unit(allpos)
    del allpos, hp, up, cl_pos
    if shuffle:
        perm = torch.randperm(ntot, generator=gen, device=device)
        pos = pos[perm]
    ids = torch.randperm(ntot, generator=gen, device=device)
    return Box(pos=pos.contiguous(), ids=ids.contiguous(), nx=nx, halo_sizes=sizes, halo_centres=centres)


def _mean_power_law(a, b, alpha):
    e1 = 1.0 - alpha
    e2 = 2.0 - alpha
    return ((b**e2 - a**e2) / e2) / ((b**e1 - a**e1) / e1)


def lattice_box(nx: int, jitter: float = 0.0, seed: int = 1, device="cpu") -> Box:
    """Uniform cell-centred lattice (optionally jittered): no seed reaches
    rho > 100, so the reference finds no halo."""
    g = torch.arange(nx, dtype=torch.float64, device=device)
    zz, yy, xx = torch.meshgrid(g, g, g, indexing="ij")
    p = torch.stack([xx, yy, zz], -1).reshape(-1, 3)
    p = (p + 0.5) / nx
    if jitter > 0:
        gen = torch.Generator(device=device)
        gen.manual_seed(seed)
        p = p + jitter / nx * (torch.rand(p.shape, generator=gen, dtype=torch.float64, device=device) - 0.5)
    pos = _to_f32_unit(p)
    ids = torch.arange(nx**3, dtype=torch.int64, device=device)
    return Box(pos=pos, ids=ids, nx=nx, halo_sizes=torch.zeros(0, dtype=torch.int64), halo_centres=torch.zeros(0, 3))


def ball_box(nx: int, centres, radii_cells, counts, seed: int = 7, background: str = "lattice", device="cpu") -> Box:
    """Uniform-density balls (radius in cells, particle count) on a uniform
    background, total particle count ``nx**3``: the analytic known-answer
    boxes (isolated halo, overlapping halos, halo across the boundary)."""
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    ntot = nx**3
    parts = []
    for c, rc, k in zip(centres, radii_cells, counts):
        u = torch.rand(k, generator=gen, dtype=torch.float64, device=device)
        r = (rc / nx) * u ** (1.0 / 3.0)
        d = _unit_vectors(gen, k, device)
        parts.append(torch.tensor(c, dtype=torch.float64, device=device) + r[:, None] * d)
    nb = sum(counts)
    nbg = ntot - nb
    bg = torch.rand(nbg, 3, generator=gen, dtype=torch.float64, device=device)
    allpos = torch.cat(parts + [bg], 0)
    pos = _to_f32_unit(allpos)
    perm = torch.randperm(ntot, generator=gen, device=device)
    pos = pos[perm].contiguous()
    ids = torch.randperm(ntot, generator=gen, device=device)
    return Box(pos=pos, ids=ids, nx=nx, halo_sizes=torch.tensor(counts), halo_centres=torch.tensor(centres))
