"""The reference's zone decomposition of the SOD stage, one GPU per rank.

The reference cuts the box into nxcpu^3 zones and gives each MPI rank a
contiguous range of them (main:321-331). For each zone a rank selects the
zone's particles with a buffer of nxbuffer cells (main:573-600), runs cic,
cicm1, tri_cic and spherover on them, keeps the halos whose centre lies in
the zone (main:2118-2120), and the ranks sum their halo counts
(main:2370). The zones need no data from one another: the buffer is
their only overlap, so there is no exchange step and no collective on the
data path, only the final count.

Results are those of the reference's P-zone run, which differ from its
one-zone run near zone edges (a halo whose particles reach beyond the
buffer, or whose seed was claimed differently); that is the reference's
own behaviour, not an approximation here.

``zones_of_rank`` restates the rank -> zone assignment, ``run_zones`` drives
one rank's zones through a zone runner (by default a ``SphericalOverdensity``
context per zone on this rank's GPU) and sums the halo counts over the
process group when one is initialised.
"""

from __future__ import annotations

from typing import Callable

import numpy as np


def zones_of_rank(rank: int, nranks: int, nzones: int) -> range:
    """The zones rank ``rank`` of ``nranks`` analyses (main:321-331): the
    first ``nzones mod nranks`` ranks take one zone more."""
    if nranks < 1 or not 0 <= rank < nranks or nzones < 0:
        raise ValueError("need 0 <= rank < nranks and nzones >= 0")
    mine = nzones // nranks
    nmod = nzones % nranks
    if rank <= nmod - 1:
        mine += 1
        first = rank * mine
        last = (rank + 1) * mine - 1
    else:
        first = rank * mine + nmod
        last = (rank + 1) * mine + nmod - 1
    return range(first, last + 1)


def gpu_zone_runner(nx: int, nxcpu: int, device: int = 0, nxbuffer: int = 0, **params) -> Callable:
    """A zone runner on one GPU: selects the zone's particles
    (``psod_select_zone``), runs the SOD stage on them in a zone context and
    returns its halo table (member indices are indices into ``pos``)."""
    import torch

    from .sod import SphericalOverdensity, select_zone

    def run(pos: np.ndarray, ids: np.ndarray, nzone: int):
        keep = select_zone(pos, nx, nxcpu, nzone, nxbuffer)
        sel = np.nonzero(keep)[0]
        with SphericalOverdensity(nx, device=device, nxcpu=nxcpu, nzone=nzone, nxbuffer=nxbuffer,
                                  **params) as s:
            s.load(torch.from_numpy(np.ascontiguousarray(pos[sel])).to(f"cuda:{device}"),
                   torch.from_numpy(np.ascontiguousarray(ids[sel])).to(f"cuda:{device}"),
                   npart_total=int(pos.shape[0]))
            s.run()
            t = s.halos()
        t.member_index = sel[t.member_index]  # back to indices into pos
        return t

    return run


def run_zones(pos: np.ndarray, ids: np.ndarray, nxcpu: int, run_zone: Callable, rank: int = 0,
              nranks: int = 1) -> tuple[dict, int]:
    """This rank's zones through ``run_zone(pos, ids, nzone) -> table`` (a
    table with ``nhalo``), and the total halo count over all ranks: the sum
    of every zone's kept halos (main:2370), all-reduced over the default
    process group when one is initialised and ``nranks > 1``."""
    tables = {z: run_zone(pos, ids, z) for z in zones_of_rank(rank, nranks, nxcpu ** 3)}
    count = sum(int(t.nhalo) for t in tables.values())
    if nranks > 1:
        import torch
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
            c = torch.tensor([count], dtype=torch.int64, device=dev)
            dist.all_reduce(c)
            count = int(c.item())
    return tables, count
