"""Host-side mirror of the reference's SOD interface.

``SphericalOverdensity`` exposes the four subroutines the Fortran driver of
sod/sod_profile_rdfof_parallel_hdf5.f90 calls (cic main:673, cicm1 main:679,
tri_cic main:713, spherover main:740) with the same argument meaning, on
top of the C-ABI in include/psod.h. Errors raise ``PsodError`` carrying the
C status (``ERR_NSEL`` / ``ERR_SELRADIUS`` keep the reference's "zone output
lost" meaning).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import capi


class PsodError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"psod status {status}: {message}")
        self.status = status


@dataclass
class HaloTable:
    halo_id: np.ndarray
    halo_mass: np.ndarray
    halo_rank: np.ndarray
    halo_center: np.ndarray
    halo_rdelta: np.ndarray
    halo_mass2: np.ndarray
    halo_mextra: np.ndarray
    halo_profile: np.ndarray
    member_offset: np.ndarray
    member_index: np.ndarray
    member_id: np.ndarray

    @property
    def nhalo(self) -> int:
        return int(self.halo_id.shape[0])


@dataclass
class FofTable:
    """Friends-of-friends catalogue (psod_fof_get_halos): halos in ascending
    ID (the ID of the lowest-index member), members in ascending input index."""

    halo_id: np.ndarray
    halo_mass: np.ndarray
    halo_com: np.ndarray
    halo_vel: np.ndarray
    halo_radius: np.ndarray
    member_offset: np.ndarray
    member_index: np.ndarray
    member_id: np.ndarray

    @property
    def nhalo(self) -> int:
        return int(self.halo_id.shape[0])

    def members(self, h: int) -> np.ndarray:
        return self.member_index[self.member_offset[h]: self.member_offset[h + 1]]


def _ptr(t):
    if t is None:
        return None
    if isinstance(t, torch.Tensor):
        return C.c_void_p(t.data_ptr())
    return C.c_void_p(t.ctypes.data)


class SphericalOverdensity:
    """One zone of the SOD stage on one GPU: the whole periodic box (the
    reference's 1-rank run) by default, or zone ``nzone`` of ``nxcpu``^3
    (``nxcpu=``, ``nzone=`` parameters) loaded with that zone's particles
    and buffer (``select_zone``)."""

    def __init__(self, nx: int, device: int = 0, **params):
        self.lib = capi.load()
        self.params = capi.default_params(nx, device=device, **params)
        h = C.c_void_p()
        st = self.lib.psod_ctx_create(C.byref(self.params), C.byref(h))
        if st != capi.OK:
            raise PsodError(st, "psod_ctx_create failed (invalid parameters or no CUDA device)")
        self.ctx = h
        self.n = 0
        # run on torch's current stream of the device: tensors torch wrote
        # are complete before the library reads them, and torch events
        # time the library's work on the same stream
        self.set_stream(torch.cuda.current_stream(device))

    # -- lifecycle -----------------------------------------------------
    def close(self):
        if getattr(self, "ctx", None):
            self.lib.psod_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int):
        if st != capi.OK:
            msg = self.lib.psod_last_error(self.ctx)
            raise PsodError(st, msg.decode() if msg else "")

    def set_stream(self, stream: torch.cuda.Stream):
        self._check(self.lib.psod_set_stream(self.ctx, C.c_void_p(stream.cuda_stream)))

    # -- the reference's entry points ---------------------------------
    def load(self, pos, ids, vel=None, npart_total: int = 0):
        """posf(3,N), idf(N), velf(3,N) of modvar (main:8-9); host or device."""
        pos = _contig(pos, torch.float32)
        ids = _contig(ids, torch.int64)
        vel = _contig(vel, torch.float32) if vel is not None else None
        n = int((pos.numel() if isinstance(pos, torch.Tensor) else pos.size) // 3)
        self.n = n
        self._keep = (pos, ids, vel)
        self._check(self.lib.psod_load_particles(self.ctx, n, _ptr(pos), _ptr(vel), _ptr(ids), int(npart_total)))

    def cic(self, want_grid: bool = False):
        """cic (main:1077-1265). Returns the (2nx)^3 grid [z,y,x] if asked."""
        grid = None
        if want_grid:
            nc = 2 * self.params.nx
            grid = np.zeros(nc**3, np.float64)
        self._check(self.lib.psod_cic(self.ctx, _ptr(grid)))
        return None if grid is None else grid.reshape(nc, nc, nc)

    def cicm1(self, want_rho: bool = True):
        """cicm1 (main:1268-1390): per-particle density, input order."""
        rho = np.zeros(self.n, np.float64) if want_rho else None
        self._check(self.lib.psod_cicm1(self.ctx, _ptr(rho)))
        return rho

    def tri_cic(self, want_isort: bool = True):
        """tri_cic (main:998-1037): (isort[:npart_new] 0-based, npart_new)."""
        nn = C.c_int64(0)
        self._check(self.lib.psod_tri_cic(self.ctx, None, C.byref(nn)))
        if not want_isort:
            return None, int(nn.value)
        isort = np.zeros(max(int(nn.value), 1), np.int64)
        self._check(self.lib.psod_tri_cic(self.ctx, _ptr(isort), C.byref(nn)))
        return isort[: int(nn.value)], int(nn.value)

    def spherover(self) -> dict:
        """spherover compute (main:1396-2201); returns run statistics."""
        st = capi.RunStats()
        self._check(self.lib.psod_spherover(self.ctx, C.byref(st)))
        return st.as_dict()

    def run(self) -> dict:
        st = capi.RunStats()
        self._check(self.lib.psod_run(self.ctx, C.byref(st)))
        return st.as_dict()

    # -- learned radius bracket ------------------------------------------
    def learn_collect(self, capacity: int):
        """Record (features, targets) of every crossing seed of later
        spherover calls (batched or learned mode); 0 stops recording."""
        self._check(self.lib.psod_learn_collect(self.ctx, int(capacity)))

    def learn_samples(self):
        """(x [n, 10], t [n, 2]) of the recorded samples, float32."""
        n = C.c_int64(0)
        self._check(self.lib.psod_learn_samples(self.ctx, C.byref(n), None, None))
        x = np.zeros((max(n.value, 1), capi.LEARN_FEATURES), np.float32)
        t = np.zeros((max(n.value, 1), 2), np.float32)
        self._check(self.lib.psod_learn_samples(self.ctx, C.byref(n), _ptr(x), _ptr(t)))
        return x[: n.value], t[: n.value]

    def learn_train(self, epochs: int = 20, batch: int = 4096, lr: float = 1e-3, seed: int = 1) -> np.ndarray:
        """Train the bracket network on the recorded samples with the
        project's GPU kernels; returns the loss of each epoch."""
        tp = capi.TrainParams(epochs=epochs, batch=batch, lr=lr, beta1=0.9, beta2=0.999, eps=1e-8, seed=seed)
        loss = np.zeros(epochs, np.float32)
        self._check(self.lib.psod_learn_train(self.ctx, C.byref(tp), _ptr(loss)))
        return loss

    def learn_get_model(self) -> np.ndarray:
        m = np.zeros(capi.LEARN_MODEL_FLOATS, np.float32)
        self._check(self.lib.psod_learn_get_model(self.ctx, _ptr(m), m.size))
        return m

    def learn_set_model(self, model):
        m = np.ascontiguousarray(model, np.float32)
        self._check(self.lib.psod_learn_set_model(self.ctx, _ptr(m), m.size))

    def learn_set_margin(self, margin: float):
        self._check(self.lib.psod_learn_set_margin(self.ctx, float(margin)))

    def learn_forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((x.shape[0], 2), np.float32)
        self._check(self.lib.psod_learn_forward(self.ctx, x.shape[0], _ptr(x), _ptr(y)))
        return y

    def learn_gradient(self, x, t):
        """(gradient over the padded parameter layout, loss) of
        0.5 * mean |y_std - t_std|^2 at the current model."""
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(capi.LEARN_PARAMS, np.float32)
        loss = C.c_float(0)
        self._check(self.lib.psod_learn_gradient(self.ctx, x.shape[0], _ptr(x), _ptr(t), _ptr(g), C.byref(loss)))
        return g, float(loss.value)

    def halo_count(self) -> tuple[int, int]:
        nh, nm = C.c_int64(0), C.c_int64(0)
        self._check(self.lib.psod_halo_count(self.ctx, C.byref(nh), C.byref(nm)))
        return int(nh.value), int(nm.value)

    def halos(self, members: bool = True, out: HaloTable | None = None) -> HaloTable:
        """The halo table of the last spherover call.  ``out`` (optional)
        supplies the arrays to fill: numpy arrays or torch tensors (pinned
        host or device), each at least as long as the table needs; the
        returned table holds views of exactly the table's length."""
        h, m = self.halo_count()
        nb = self.params.nbins
        ne = self.params.ndelta_extra
        if out is not None:
            need = dict(halo_id=h, halo_mass=h, halo_rank=h, halo_center=3 * h, halo_rdelta=h, halo_mass2=h,
                        halo_mextra=h * ne, halo_profile=h * nb, member_offset=h + 1,
                        member_index=m if members else 0, member_id=m if members else 0)
            views = {}
            for f, k in need.items():
                a = getattr(out, f)
                flat = a.reshape(-1)
                if flat.shape[0] < k:
                    raise ValueError(f"halos(out=...): {f} holds {flat.shape[0]} entries, needs {k}")
                views[f] = flat[:k]
            ct = capi.HaloTable()
            for f, _ in capi.HaloTable._fields_:
                v = views[f]
                setattr(ct, f, None if v.shape[0] == 0 else _ptr(v).value)
            self._check(self.lib.psod_get_halos(self.ctx, C.byref(ct)))
            views["halo_center"] = views["halo_center"].reshape(h, 3)
            views["halo_mextra"] = views["halo_mextra"].reshape(h, ne)
            views["halo_profile"] = views["halo_profile"].reshape(h, nb)
            return HaloTable(**views)
        t = HaloTable(
            halo_id=np.zeros(h, np.int64),
            halo_mass=np.zeros(h, np.int64),
            halo_rank=np.zeros(h, np.int64),
            halo_center=np.zeros((h, 3), np.float32),
            halo_rdelta=np.zeros(h, np.float64),
            halo_mass2=np.zeros(h, np.int64),
            halo_mextra=np.zeros((h, ne), np.int64),
            halo_profile=np.zeros((h, nb), np.int64),
            member_offset=np.zeros(h + 1, np.int64),
            member_index=np.zeros(m if members else 0, np.int64),
            member_id=np.zeros(m if members else 0, np.int64),
        )
        ct = capi.HaloTable()
        for f, _ in capi.HaloTable._fields_:
            a = getattr(t, f)
            if f.startswith("member_") and f != "member_offset" and not members:
                setattr(ct, f, None)
            elif a.size == 0:
                setattr(ct, f, None)
            else:
                setattr(ct, f, a.ctypes.data)
        self._check(self.lib.psod_get_halos(self.ctx, C.byref(ct)))
        return t


    # ---- scheduling thresholds (no effect on any result) ----
    def get_tuning(self) -> dict:
        t = capi.Tuning()
        self._check(self.lib.psod_get_tuning(self.ctx, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = capi.Tuning(**{**self.get_tuning(), **kw})
        self._check(self.lib.psod_set_tuning(self.ctx, C.byref(t)))

    def autotune(self) -> dict:
        """Time psod_spherover over a few threshold candidates on the loaded
        particles (after tri_cic) and keep the fastest (psod_autotune)."""
        t, ms, n = capi.Tuning(), C.c_double(0.0), C.c_int32(0)
        self._check(self.lib.psod_autotune(self.ctx, C.byref(t), C.byref(ms), C.byref(n)))
        return dict(t.as_dict(), ms_best=ms.value, runs=n.value)

    # ---- friends-of-friends (pFoF fofpara + merge + modhalo observables) ----
    def fof(self, percolation: float = 0.2, mmin: int = 20, nres: int = 0) -> dict:
        """pFoF's halo finder on the loaded particles (one rank, periodic
        box): modfofpara.f90 fofpara with the modfofmpi.f90 merge, then
        selecthaloes / computecom / computeradius.  ``percolation`` is
        param%percolation_length, ``mmin`` param%Mmin, ``nres`` the
        particles per side (0: cube root of the count).  Returns the
        counters; the catalogue comes from fof_halos()."""
        p = capi.FofParams(percolation, 0, nres, mmin)
        st = capi.FofStats()
        self._check(self.lib.psod_fof(self.ctx, C.byref(p), C.byref(st)))
        return st.as_dict()

    def fof_release(self):
        """Free the FoF stage's working arrays (the catalogue stays)."""
        self._check(self.lib.psod_fof_release(self.ctx))

    def learn_set_features(self, which: str):
        """The learned bracket's feature set: "seed" (seed-local) or "fof"
        (from the seed's FoF group; needs fof() on the loaded particles)."""
        self._check(self.lib.psod_learn_set_features(
            self.ctx, capi.LEARN_FEATURES_FOF if which == "fof" else capi.LEARN_FEATURES_SEED))

    def fof_halos(self, members: bool = True) -> FofTable:
        nh, nm = C.c_int64(0), C.c_int64(0)
        self._check(self.lib.psod_fof_halo_count(self.ctx, C.byref(nh), C.byref(nm)))
        h, m = int(nh.value), int(nm.value)
        t = FofTable(halo_id=np.zeros(h, np.int64), halo_mass=np.zeros(h, np.int64),
                     halo_com=np.zeros((h, 3), np.float64), halo_vel=np.zeros((h, 3), np.float64),
                     halo_radius=np.zeros(h, np.float64), member_offset=np.zeros(h + 1, np.int64),
                     member_index=np.zeros(m if members else 0, np.int64),
                     member_id=np.zeros(m if members else 0, np.int64))
        ct = capi.FofTable()
        for f, _ in capi.FofTable._fields_:
            a = getattr(t, f)
            setattr(ct, f, None if a.size == 0 else a.ctypes.data)
        self._check(self.lib.psod_fof_get_halos(self.ctx, C.byref(ct)))
        return t


    # ---- halo properties (haloanalyzer's halo_properties) ----
    def halo_properties(self, unit_l: float, unit_d: float, unit_t: float, aexp: float, h0: float, hz: float,
                        delta_vir: float, levelmin: int, source: str = "sod", center_on_mass: bool = False,
                        periodic: bool = True, epot_threshold: int = 30000) -> tuple[dict, dict]:
        """haloanalyzer_new/src/modfunctions.f90 halo_properties for every
        halo of the last SOD table (``source="sod"``) or FoF catalogue
        (``source="fof"``).  Returns (properties, counters): each property an
        array of shape (nhalo,) or (nhalo, k) in the reference's units and
        precision."""
        p = capi.PropsParams(unit_l, unit_d, unit_t, aexp, h0, hz, delta_vir, levelmin, int(center_on_mass),
                             int(periodic), capi.PROPS_FROM_FOF if source == "fof" else capi.PROPS_FROM_SOD,
                             epot_threshold, 0)
        st = capi.PropsStats()
        self._check(self.lib.psod_halo_properties(self.ctx, C.byref(p), C.byref(st)))
        nh = int(st.nhalo)
        out = {f: np.zeros((nh, k) if k > 1 else nh, dtype=dt) for f, k, dt in capi.PROPS_FIELDS}
        ct = capi.PropsTable()
        for f, _, _ in capi.PROPS_FIELDS:
            setattr(ct, f, None if out[f].size == 0 else out[f].ctypes.data)
        self._check(self.lib.psod_props_get(self.ctx, C.byref(ct)))
        return out, st.as_dict()


def _host_table(t: HaloTable) -> tuple[capi.HaloTable, list]:
    """A C halo table pointing at host numpy copies of ``t``'s arrays (the
    copies are returned too, to keep them alive during the call)."""
    keep = []
    ct = capi.HaloTable()
    dtypes = dict(halo_center=np.float32, halo_rdelta=np.float64)
    for f, _ in capi.HaloTable._fields_:
        a = getattr(t, f)
        if isinstance(a, torch.Tensor):
            a = a.detach().cpu().numpy()
        a = np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=dtypes.get(f, np.int64))
        keep.append(a)
        setattr(ct, f, None if a.size == 0 else a.ctypes.data)
    return ct, keep


def write_masst(path: str, table: HaloTable) -> None:
    """The reference's "masst" file of one zone (main:2234-2239): Fortran
    unformatted records of namas, then (ID, N_delta, centre) per halo."""
    lib = capi.load()
    ct, keep = _host_table(table)
    st = lib.psod_write_masst(str(path).encode(), C.byref(ct), table.nhalo)
    if st != capi.OK:
        raise PsodError(st, f"psod_write_masst({path}) failed")


def write_strct(path: str, table: HaloTable, pos, ids, vel=None, pot=None, force=None) -> None:
    """The reference's "strct" file of one zone (main:2246-2256): per halo
    N_delta, then its members' positions, velocities, IDs (and potential /
    force when given), members in ascending distance.  ``pos``/``vel``/
    ``ids`` are the zone's particle arrays in input order."""
    lib = capi.load()
    ct, keep = _host_table(table)

    def host(a, dt, width):
        if a is None:
            return None
        if isinstance(a, torch.Tensor):
            a = a.detach().cpu().numpy()
        return np.ascontiguousarray(np.asarray(a, dtype=dt).reshape(-1, width) if width > 1 else
                                    np.asarray(a, dtype=dt).reshape(-1))

    p, i = host(pos, np.float32, 3), host(ids, np.int64, 1)
    v, q, fo = host(vel, np.float32, 3), host(pot, np.float32, 1), host(force, np.float32, 3)
    n = i.shape[0]
    st = lib.psod_write_strct(str(path).encode(), C.byref(ct), table.nhalo, n, _ptr(p), _ptr(v), _ptr(i), _ptr(q),
                              _ptr(fo))
    if st != capi.OK:
        raise PsodError(st, f"psod_write_strct({path}) failed")


def _contig(x, dtype):
    if isinstance(x, torch.Tensor):
        return x.to(dtype).contiguous()
    return np.ascontiguousarray(x, dtype=torch.empty(0, dtype=dtype).numpy().dtype)


def read_cube_zone(root: str, ncpu: int, nzone: int, nx: int, nxbuffer: int = 0, id_bytes: int = 8):
    """The reference's binary particle reader (main:455-534): the particles
    of zone ``nzone`` from the cube files ``<root>_cube_NNNNN`` of an
    ``ncpu``-cube decomposition, as (pos (n, 3) float32 box units, vel (n, 3)
    float32, ids int64) in the reference's order, ready for ``load``."""
    lib = capi.load()
    n = C.c_int64(0)
    st = lib.psod_read_cube_zone(str(root).encode(), ncpu, nzone, nx, nxbuffer, id_bytes, 0, C.byref(n), None, None,
                                 None)
    if st != capi.OK:
        raise PsodError(st, f"psod_read_cube_zone({root}, zone {nzone}) failed")
    pos = np.zeros((max(n.value, 1), 3), np.float32)
    vel = np.zeros((max(n.value, 1), 3), np.float32)
    ids = np.zeros(max(n.value, 1), np.int64)
    st = lib.psod_read_cube_zone(str(root).encode(), ncpu, nzone, nx, nxbuffer, id_bytes, pos.shape[0], C.byref(n),
                                 _ptr(pos), _ptr(vel), _ptr(ids))
    if st != capi.OK:
        raise PsodError(st, f"psod_read_cube_zone({root}, zone {nzone}) failed")
    return pos[: n.value], vel[: n.value], ids[: n.value]


def select_zone(pos, nx: int, nxcpu: int, nzone: int, nxbuffer: int = 0) -> np.ndarray:
    """The driver's selection of one zone's particles with their buffer
    (main:573-600) through ``psod_select_zone``: a boolean mask over ``pos``
    ((n, 3) float32, box units) of the particles that a context with
    ``nxcpu=nxcpu, nzone=nzone`` is loaded with, in input order."""
    lib = capi.load()
    pos = np.ascontiguousarray(pos, np.float32)
    n = pos.shape[0]
    keep = np.zeros(max(n, 1), np.uint8)
    nk = C.c_int64(0)
    st = lib.psod_select_zone(nx, nxcpu, nzone, nxbuffer, _ptr(pos), n, _ptr(keep), C.byref(nk))
    if st != capi.OK:
        raise PsodError(st, f"psod_select_zone(nx={nx}, nxcpu={nxcpu}, nzone={nzone}) failed")
    return keep[:n].astype(bool)

