"""ctypes wrapper of the CPU oracle (test infrastructure only).

TEST INFRASTRUCTURE: used by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg as the checker; the product never imports it.

The oracle restates the 1-rank SOD stage of
sod/sod_profile_rdfof_parallel_hdf5.f90 (cic main:1077-1265, cicm1
main:1268-1390, tri_cic main:998-1037, quick_sort main:2477-2571,
spherover main:1396-2201). Parity unpinned: the reference has no golden
vectors for this path.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpsod_oracle.so")

REFERENCE = 0
CANONICAL = 1
MAX_EXTRA = 4


class _Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("nmin", C.c_int32),
        ("delta", C.c_double),
        ("delta2", C.c_double),
        ("ncut", C.c_int32),
        ("nsel", C.c_int64),
        ("nxbuffer", C.c_int32),
        ("nbins", C.c_int32),
        ("rbin_lo", C.c_double),
        ("rbin_hi", C.c_double),
        ("ndelta_extra", C.c_int32),
        ("delta_extra", C.c_double * MAX_EXTRA),
        ("npart_total", C.c_int64),
        ("nxcpu", C.c_int32),
        ("nzone", C.c_int32),
    ]


class _Result(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("fail_rank", C.c_int64),
        ("npart_new", C.c_int64),
        ("nprocessed", C.c_int64),
        ("cross_touch", C.c_int64),
        ("nhalo", C.c_int64),
        ("nmember", C.c_int64),
        ("halo_id", C.POINTER(C.c_int64)),
        ("halo_mass", C.POINTER(C.c_int64)),
        ("halo_rank", C.POINTER(C.c_int64)),
        ("halo_cidx", C.POINTER(C.c_int64)),
        ("halo_center", C.POINTER(C.c_float)),
        ("halo_rdelta", C.POINTER(C.c_double)),
        ("halo_mass2", C.POINTER(C.c_int64)),
        ("halo_mextra", C.POINTER(C.c_int64)),
        ("halo_profile", C.POINTER(C.c_int64)),
        ("member_offset", C.POINTER(C.c_int64)),
        ("member_index", C.POINTER(C.c_int64)),
    ]


class _Audit(C.Structure):
    _fields_ = [
        ("refine_seeds", C.c_int64),
        ("refine_flips", C.c_int64),
        ("refine_near", C.c_int64),
        ("dist_tie_cut", C.c_int64),
        ("dist_tie_cut_nmax", C.c_int64),
        ("dist_tie_members", C.c_int64),
    ]


_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.psod_oracle_quick_sort.argtypes = [P(C.c_double), P(C.c_int64), C.c_int64]
        L.psod_oracle_cic.argtypes = [P(_Params), C.c_int64, P(C.c_float), C.c_int, P(C.c_double)]
        L.psod_oracle_cicm1.argtypes = [P(_Params), C.c_int64, P(C.c_float), P(C.c_double), P(C.c_double)]
        L.psod_oracle_tri_cic.argtypes = [C.c_int64, P(C.c_double), C.c_int, P(C.c_int64), P(C.c_int64)]
        L.psod_oracle_run.argtypes = [P(_Params), C.c_int64, P(C.c_float), P(C.c_int64), C.c_int, P(_Result)]
        L.psod_oracle_spherover.argtypes = [
            P(_Params), C.c_int64, P(C.c_float), P(C.c_int64), P(C.c_int64), C.c_int64, C.c_int, P(_Result)
        ]
        L.psod_oracle_audit_spherover.argtypes = [
            P(_Params), C.c_int64, P(C.c_float), P(C.c_int64), P(C.c_int64), C.c_int64, C.c_int, P(_Result), P(_Audit)
        ]
        L.psod_oracle_free.argtypes = [P(_Result)]
        _lib = L
    return _lib


@dataclass
class Params:
    """Same meaning and defaults as the reference CLI (main:110-114, 1414)."""

    nx: int
    nmin: int = 100
    delta: float = 200.0
    delta2: float = 800.0
    ncut: int = 4
    nsel: int = 4_000_000
    nxbuffer: int = 0
    nbins: int = 60
    rbin_lo: float = 0.01
    rbin_hi: float = 1.0
    delta_extra: tuple = ()
    npart_total: int = 0
    nxcpu: int = 1  # zones per axis (nxcpu^3 zones, main:340-342)
    nzone: int = 0  # zone analysed, z fastest (main:344-346)

    def c(self, n: int) -> _Params:
        p = _Params()
        p.nx = self.nx
        p.nmin = self.nmin
        p.delta = self.delta
        p.delta2 = self.delta2
        p.ncut = self.ncut
        p.nsel = self.nsel
        p.nxbuffer = self.nxbuffer
        p.nbins = self.nbins
        p.rbin_lo = self.rbin_lo
        p.rbin_hi = self.rbin_hi
        p.ndelta_extra = len(self.delta_extra)
        for i, d in enumerate(self.delta_extra):
            p.delta_extra[i] = d
        p.npart_total = self.npart_total if self.npart_total > 0 else n
        p.nxcpu = self.nxcpu
        p.nzone = self.nzone
        return p


@dataclass
class Result:
    status: int
    fail_rank: int
    npart_new: int
    nprocessed: int
    cross_touch: int = 0
    halo_id: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    halo_mass: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    halo_rank: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    halo_cidx: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    halo_center: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    halo_rdelta: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    halo_mass2: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    halo_mextra: np.ndarray = field(default_factory=lambda: np.zeros((0, 0), np.int64))
    halo_profile: np.ndarray = field(default_factory=lambda: np.zeros((0, 0), np.int64))
    member_offset: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int64))
    member_index: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))

    @property
    def nhalo(self) -> int:
        return int(self.halo_id.shape[0])


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def _as_pos(pos) -> np.ndarray:
    a = pos.cpu().numpy() if hasattr(pos, "cpu") else np.asarray(pos)
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1, 3)


def _as_ids(ids) -> np.ndarray:
    a = ids.cpu().numpy() if hasattr(ids, "cpu") else np.asarray(ids)
    return np.ascontiguousarray(a, dtype=np.int64)


def quick_sort(values) -> tuple[np.ndarray, np.ndarray]:
    lst = np.ascontiguousarray(values, dtype=np.float64).copy()
    order = np.zeros(lst.shape[0], np.int64)
    lib().psod_oracle_quick_sort(_ptr(lst, C.c_double), _ptr(order, C.c_int64), lst.shape[0])
    return lst, order


def cic_grid(params: Params, pos, mode=REFERENCE) -> np.ndarray:
    p = _as_pos(pos)
    nc = 2 * params.nx
    grid = np.zeros(nc**3, np.float64)
    cp = params.c(p.shape[0])
    st = lib().psod_oracle_cic(C.byref(cp), p.shape[0], _ptr(p, C.c_float), mode, _ptr(grid, C.c_double))
    if st:
        raise ValueError(f"oracle cic status {st}")
    return grid.reshape(nc, nc, nc)  # [z, y, x]


def rho(params: Params, pos, mode=REFERENCE, grid=None) -> np.ndarray:
    p = _as_pos(pos)
    if grid is None:
        grid = cic_grid(params, p, mode)
    g = np.ascontiguousarray(grid, dtype=np.float64).reshape(-1)
    out = np.zeros(p.shape[0], np.float64)
    cp = params.c(p.shape[0])
    st = lib().psod_oracle_cicm1(C.byref(cp), p.shape[0], _ptr(p, C.c_float), _ptr(g, C.c_double), _ptr(out, C.c_double))
    if st:
        raise ValueError(f"oracle cicm1 status {st}")
    return out


def tri_cic(rho_values, mode=REFERENCE) -> tuple[np.ndarray, int]:
    r = np.ascontiguousarray(rho_values, dtype=np.float64)
    isort = np.zeros(r.shape[0], np.int64)
    nn = C.c_int64(0)
    lib().psod_oracle_tri_cic(r.shape[0], _ptr(r, C.c_double), mode, _ptr(isort, C.c_int64), C.byref(nn))
    return isort, int(nn.value)


def _collect(res: _Result, params: Params) -> Result:
    out = Result(status=res.status, fail_rank=res.fail_rank, npart_new=res.npart_new, nprocessed=res.nprocessed,
                 cross_touch=res.cross_touch)
    h = int(res.nhalo)
    if res.status == 0:
        def arr(ptr, n, dt):
            if n == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(ptr, shape=(n,)).copy().astype(dt)

        out.halo_id = arr(res.halo_id, h, np.int64)
        out.halo_mass = arr(res.halo_mass, h, np.int64)
        out.halo_rank = arr(res.halo_rank, h, np.int64)
        out.halo_cidx = arr(res.halo_cidx, h, np.int64)
        out.halo_center = arr(res.halo_center, 3 * h, np.float32).reshape(h, 3)
        out.halo_rdelta = arr(res.halo_rdelta, h, np.float64)
        out.halo_mass2 = arr(res.halo_mass2, h, np.int64)
        ne = len(params.delta_extra)
        out.halo_mextra = arr(res.halo_mextra, ne * h, np.int64).reshape(h, ne)
        out.halo_profile = arr(res.halo_profile, params.nbins * h, np.int64).reshape(h, params.nbins)
        out.member_offset = arr(res.member_offset, h + 1, np.int64)
        out.member_index = arr(res.member_index, int(res.nmember), np.int64)
    return out


def zone_select(pos, nx: int, nxcpu: int, nzone: int, nxbuffer: int = 0) -> np.ndarray:
    """The driver's selection of zone ``nzone``'s particles with their
    buffer (main:573-600): zone indices as main:344-346, centre as
    main:428-430, half-widths rxsmall/rxlarge as main:433-439, and on every
    axis |x - xc| < rxsmall or > rxlarge in FP64 (main:578-584)."""
    p = np.asarray(pos, dtype=np.float32).reshape(-1, 3).astype(np.float64)
    ncpu = nxcpu
    ix = int(nzone / float(ncpu * ncpu))
    iy = int((nzone - ix * ncpu * ncpu) / float(ncpu))
    iz = nzone - ix * ncpu * ncpu - iy * ncpu
    nxzone = nx // ncpu
    nxb = nxbuffer if nxbuffer != 0 else nxzone // 2
    keep = np.ones(p.shape[0], dtype=bool)
    for a, i in enumerate((ix, iy, iz)):
        lo, hi = i / float(ncpu), (i + 1) / float(ncpu)
        xc = (lo + hi) / 2.0
        rs = (0.5 + nxb / float(nxzone)) / float(ncpu)
        rl = 1.0 - rs
        d = np.abs(p[:, a] - xc)
        keep &= (d < rs) | (d > rl)
    return keep


def run(params: Params, pos, ids, mode=REFERENCE) -> Result:
    """cic -> cicm1 -> tri_cic -> spherover for one zone (``params.nxcpu``,
    ``params.nzone``; the whole box by default) on the particles given."""
    p = _as_pos(pos)
    i = _as_ids(ids)
    cp = params.c(p.shape[0])
    res = _Result()
    lib().psod_oracle_run(C.byref(cp), p.shape[0], _ptr(p, C.c_float), _ptr(i, C.c_int64), mode, C.byref(res))
    try:
        return _collect(res, params)
    finally:
        lib().psod_oracle_free(C.byref(res))


def spherover(params: Params, pos, ids, isort, npart_new, mode=REFERENCE) -> Result:
    p = _as_pos(pos)
    i = _as_ids(ids)
    s = np.ascontiguousarray(isort, dtype=np.int64)
    cp = params.c(p.shape[0])
    res = _Result()
    lib().psod_oracle_spherover(
        C.byref(cp), p.shape[0], _ptr(p, C.c_float), _ptr(i, C.c_int64), _ptr(s, C.c_int64), npart_new, mode, C.byref(res)
    )
    try:
        return _collect(res, params)
    finally:
        lib().psod_oracle_free(C.byref(res))


def audit_spherover(params: Params, pos, ids, isort, npart_new, mode=REFERENCE) -> tuple[Result, dict]:
    """spherover in ``mode`` with the refinement evaluated in both
    arithmetics side by side; returns the result and the audit counters."""
    p = _as_pos(pos)
    i = _as_ids(ids)
    s = np.ascontiguousarray(isort, dtype=np.int64)
    cp = params.c(p.shape[0])
    res = _Result()
    au = _Audit()
    lib().psod_oracle_audit_spherover(
        C.byref(cp), p.shape[0], _ptr(p, C.c_float), _ptr(i, C.c_int64), _ptr(s, C.c_int64), npart_new, mode,
        C.byref(res), C.byref(au)
    )
    try:
        return _collect(res, params), {f: int(getattr(au, f)) for f, _ in _Audit._fields_}
    finally:
        lib().psod_oracle_free(C.byref(res))


def arithmetic_audit(params: Params, pos, ids) -> dict:
    """Where the reference's FP64 arithmetic and quicksort tie orders and the
    canonical arithmetic (int64 fixed point, index tie-breaks) of the GPU
    part ways on one box, step by step:
      rho_differ          particles whose rho differs (FP64 file-order sums vs
                          fixed point; relative gaps ~1e-16)
      seed_order_moved    seed ranks holding a different particle
      seed_adjacent_swaps neighbouring seed pairs exchanged
      seed_exact_ties     neighbouring seeds with exactly equal 1/rho (either
                          arithmetic)
      refine_*            from the reference run: seeds whose FP64-sum and
                          fixed-point-sum argmax differ, seeds whose best two
                          fixed-point sums are within 1e-9
      dist_tie_*          crossings with exactly equal distances at the
                          N_delta cut / among the members
      halos_*             the two full runs compared halo by halo (matched by
                          centre particle ID): halos in one run only, equal
                          centres with a different N_delta, R_delta or member
                          set."""
    p = _as_pos(pos)
    i = _as_ids(ids)
    r_ref = rho(params, p, REFERENCE)
    r_can = rho(params, p, CANONICAL)
    s_ref, n_ref = tri_cic(r_ref, REFERENCE)
    s_can, n_can = tri_cic(r_can, CANONICAL)
    nn = min(n_ref, n_can)
    moved = int(np.count_nonzero(s_ref[:nn] != s_can[:nn]))
    swaps = int(np.count_nonzero((s_ref[: nn - 1] == s_can[1:nn]) & (s_ref[1:nn] == s_can[: nn - 1])))
    pd_ref = 1.0 / r_ref[s_ref[:n_ref]]
    pd_can = 1.0 / r_can[s_can[:n_can]]
    ties = int(np.count_nonzero(pd_ref[1:] == pd_ref[:-1])) + int(np.count_nonzero(pd_can[1:] == pd_can[:-1]))
    res_ref, au = audit_spherover(params, p, i, s_ref, n_ref, REFERENCE)
    res_can = spherover(params, p, i, s_can, n_can, CANONICAL)
    out = dict(rho_differ=int(np.count_nonzero(r_ref != r_can)),
               rho_max_rel=float(np.max(np.abs(r_ref - r_can) / np.maximum(np.abs(r_ref), 1e-300))),
               npart_new=(n_ref, n_can), seed_order_moved=moved, seed_adjacent_swaps=swaps, seed_exact_ties=ties,
               refine_seeds=au["refine_seeds"], refine_flips=au["refine_flips"], refine_near=au["refine_near"],
               dist_tie_cut=au["dist_tie_cut"], dist_tie_cut_nmax=au["dist_tie_cut_nmax"],
               dist_tie_members=au["dist_tie_members"],
               status=(res_ref.status, res_can.status), nhalo=(res_ref.nhalo, res_can.nhalo))
    a = {int(h): k for k, h in enumerate(res_ref.halo_id)}
    b = {int(h): k for k, h in enumerate(res_can.halo_id)}
    only = len(set(a) ^ set(b))
    dmass = drad = dset = 0
    for h in set(a) & set(b):
        x, y = a[h], b[h]
        if res_ref.halo_mass[x] != res_can.halo_mass[y]:
            dmass += 1
        if res_ref.halo_rdelta[x] != res_can.halo_rdelta[y]:
            drad += 1
        mx = res_ref.member_index[res_ref.member_offset[x]: res_ref.member_offset[x + 1]]
        my = res_can.member_index[res_can.member_offset[y]: res_can.member_offset[y + 1]]
        if not np.array_equal(np.sort(mx), np.sort(my)):
            dset += 1
    out.update(halos_one_run_only=only, halos_mass_differ=dmass, halos_rdelta_differ=drad,
               halos_members_differ=dset)
    return out


# ---------------------------------------------------------------------------
# friends-of-friends (pFoF fofpara + periodic merge + sod/modhalo.f90
# selecthaloes, computecom, computeradius; psod_oracle_fof.c)
# ---------------------------------------------------------------------------
class _FofParams(C.Structure):
    _fields_ = [("percolation", C.c_float), ("nres", C.c_int64), ("mmin", C.c_int64)]


class _FofResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("ngroups_local", C.c_int64),
        ("nbridges", C.c_int64),
        ("nhalo", C.c_int64),
        ("nmember", C.c_int64),
        ("halo_id", C.POINTER(C.c_int64)),
        ("halo_mass", C.POINTER(C.c_int64)),
        ("halo_com", C.POINTER(C.c_double)),
        ("halo_vel", C.POINTER(C.c_double)),
        ("halo_radius", C.POINTER(C.c_double)),
        ("member_offset", C.POINTER(C.c_int64)),
        ("member_index", C.POINTER(C.c_int64)),
        ("structure", C.POINTER(C.c_int64)),
    ]


@dataclass
class FofResult:
    """The reference's FoF catalogue: halos in ascending label, members in
    heap order inside a halo, plus every particle's final label."""

    status: int
    ngroups_local: int = 0
    nbridges: int = 0
    halo_id: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    halo_mass: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    halo_com: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float64))
    halo_vel: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float64))
    halo_radius: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    member_offset: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int64))
    member_index: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    structure: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))

    @property
    def nhalo(self) -> int:
        return int(self.halo_id.shape[0])

    def members(self, h: int) -> np.ndarray:
        return self.member_index[self.member_offset[h]: self.member_offset[h + 1]]


def fof(pos, ids, vel=None, percolation: float = 0.2, nres: int | None = None, mmin: int = 20) -> FofResult:
    """pFoF on one rank over the periodic unit box (modfofpara.f90:31-296,
    modfofmpi.f90:37-649, sod/modhalo.f90:253-488)."""
    L = lib()
    if not hasattr(L, "_fof_ready"):
        L.psod_oracle_fof.argtypes = [C.POINTER(_FofParams), C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                      C.POINTER(C.c_int64), C.POINTER(_FofResult)]
        L.psod_oracle_fof_free.argtypes = [C.POINTER(_FofResult)]
        L._fof_ready = True
    p = _as_pos(pos)
    i = _as_ids(ids)
    n = p.shape[0]
    if nres is None:
        nres = int(round(n ** (1.0 / 3.0)))
    v = None if vel is None else np.ascontiguousarray(
        vel.cpu().numpy() if hasattr(vel, "cpu") else vel, dtype=np.float32).reshape(-1, 3)
    cp = _FofParams(percolation, nres, mmin)
    r = _FofResult()
    st = L.psod_oracle_fof(C.byref(cp), n, _ptr(p, C.c_float), None if v is None else _ptr(v, C.c_float),
                           _ptr(i, C.c_int64), C.byref(r))
    if st != 0:
        L.psod_oracle_fof_free(C.byref(r))
        return FofResult(status=st)
    nh, nm = r.nhalo, r.nmember

    def take(ptr, count, dtype, shape=None):
        a = np.ctypeslib.as_array(ptr, shape=(max(count, 1),))[:count].astype(dtype, copy=True)
        return a.reshape(shape) if shape else a

    out = FofResult(status=0, ngroups_local=r.ngroups_local, nbridges=r.nbridges,
                    halo_id=take(r.halo_id, nh, np.int64), halo_mass=take(r.halo_mass, nh, np.int64),
                    halo_com=take(r.halo_com, 3 * nh, np.float64, (nh, 3)),
                    halo_vel=take(r.halo_vel, 3 * nh, np.float64, (nh, 3)),
                    halo_radius=take(r.halo_radius, nh, np.float64),
                    member_offset=take(r.member_offset, nh + 1, np.int64),
                    member_index=take(r.member_index, nm, np.int64),
                    structure=take(r.structure, n, np.int64))
    L.psod_oracle_fof_free(C.byref(r))
    return out


# ---------------------------------------------------------------------------
# halo properties (haloanalyzer halo_properties; psod_oracle_props.c)
# ---------------------------------------------------------------------------
PROPS_NBIN1 = 100
PROPS_NBIN2 = 30


class _PropsParams(C.Structure):
    _fields_ = [("unit_l", C.c_double), ("unit_d", C.c_double), ("unit_t", C.c_double), ("aexp", C.c_double),
                ("h0", C.c_double), ("hz", C.c_double), ("delta_vir", C.c_double), ("levelmin", C.c_int32),
                ("center_on_mass", C.c_int32), ("periodic", C.c_int32), ("epot_threshold", C.c_int32)]


_PROPS_OUT = [
    ("npart", 1, np.int64), ("mvir", 1, np.float64), ("rvir", 1, np.float64), ("rvircom", 1, np.float64),
    ("vvir", 1, np.float64), ("com", 3, np.float32), ("comv", 3, np.float32), ("rmax", 1, np.float32),
    ("vmax", 1, np.float32), ("dispx", 1, np.float32), ("dispv", 1, np.float32), ("ekin", 1, np.float32),
    ("epot", 1, np.float32), ("lambda", 3, np.float32), ("lambda_prime", 3, np.float32),
    ("eig_val", 3, np.float32), ("eig_vec", 3, np.float32), ("cos_alpha", 1, np.float64),
    ("center_pot", 3, np.float32), ("circ", 4, np.float32), ("delta_vals", 2, np.float32),
    ("dens", PROPS_NBIN1, np.float32), ("dens_int", PROPS_NBIN1, np.float32), ("vcirc", PROPS_NBIN1, np.float32),
    ("dens178", PROPS_NBIN2, np.float32), ("dens_int178", PROPS_NBIN2, np.float32),
]


class _PropsOut(C.Structure):
    _fields_ = [(f, C.c_void_p) for f, _, _ in _PROPS_OUT]


def halo_properties(offset, member, pos, vel=None, *, unit_l, unit_d, unit_t, aexp, h0, hz, delta_vir, levelmin,
                    center_on_mass=False, periodic=True, epot_threshold=30000) -> dict:
    """haloanalyzer_new/src/modfunctions.f90 halo_properties (:47-808) for
    halos given as member lists (offset[h]..offset[h+1] into member, input
    indices into pos / vel), in the reference's statement order."""
    L = lib()
    if not hasattr(L, "_props_ready"):
        L.psod_oracle_halo_properties.argtypes = [C.POINTER(_PropsParams), C.c_int64, C.POINTER(C.c_int64),
                                                  C.POINTER(C.c_int64), C.POINTER(C.c_float),
                                                  C.POINTER(C.c_float), C.POINTER(_PropsOut)]
        L._props_ready = True
    off = np.ascontiguousarray(offset, np.int64)
    mem = np.ascontiguousarray(member, np.int64)
    p = _as_pos(pos)
    v = None if vel is None else np.ascontiguousarray(
        vel.cpu().numpy() if hasattr(vel, "cpu") else vel, dtype=np.float32).reshape(-1, 3)
    nh = off.shape[0] - 1
    out = {f: np.zeros((nh, k) if k > 1 else nh, dtype=dt) for f, k, dt in _PROPS_OUT}
    co = _PropsOut(*[out[f].ctypes.data if out[f].size else None for f, _, _ in _PROPS_OUT])
    cp = _PropsParams(unit_l, unit_d, unit_t, aexp, h0, hz, delta_vir, levelmin, int(center_on_mass), int(periodic),
                      epot_threshold)
    st = L.psod_oracle_halo_properties(C.byref(cp), nh, _ptr(off, C.c_int64), _ptr(mem, C.c_int64),
                                       _ptr(p, C.c_float), None if v is None else _ptr(v, C.c_float), C.byref(co))
    if st != 0:
        raise ValueError(f"psod_oracle_halo_properties status {st}")
    return out
