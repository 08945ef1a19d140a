"""ctypes binding of libpsod.so (include/psod.h).

The product path: every call goes to the sm_100a kernels in the in-tree
library. There is no CPU fallback; without the library or a CUDA device the
calls raise.
"""

from __future__ import annotations

import ctypes as C
import os

from . import build as _build

MAX_EXTRA = 4

OK = 0
ERR_NSEL = 1
ERR_SELRADIUS = 2
ERR_TIMEOUT = 3
ERR_CUDA = 4
ERR_ARG = 5
ERR_STATE = 6
ERR_NOMEM = 7
ERR_IO = 8

MODE_PLAIN = 0
MODE_BATCHED = 1
MODE_LEARNED = 2

LEARN_FEATURES_SEED = 0
LEARN_FEATURES_FOF = 1


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("nmin", C.c_int32),
        ("delta", C.c_double),
        ("delta2", C.c_double),
        ("ncut", C.c_int32),
        ("nsel", C.c_int64),
        ("nxbuffer", C.c_int32),
        ("npu", C.c_int64),
        ("nbins", C.c_int32),
        ("rbin_lo", C.c_double),
        ("rbin_hi", C.c_double),
        ("ndelta_extra", C.c_int32),
        ("delta_extra", C.c_double * MAX_EXTRA),
        ("mode", C.c_int32),
        ("device", C.c_int32),
        ("nxcpu", C.c_int32),
        ("nzone", C.c_int32),
    ]


class HaloTable(C.Structure):
    _fields_ = [
        ("halo_id", C.c_void_p),
        ("halo_mass", C.c_void_p),
        ("halo_rank", C.c_void_p),
        ("halo_center", C.c_void_p),
        ("halo_rdelta", C.c_void_p),
        ("halo_mass2", C.c_void_p),
        ("halo_mextra", C.c_void_p),
        ("halo_profile", C.c_void_p),
        ("member_offset", C.c_void_p),
        ("member_index", C.c_void_p),
        ("member_id", C.c_void_p),
    ]


class RunStats(C.Structure):
    _fields_ = [
        ("npart_new", C.c_int64),
        ("nprocessed", C.c_int64),
        ("nhalo", C.c_int64),
        ("nmember", C.c_int64),
        ("rounds", C.c_int64),
        ("fail_rank", C.c_int64),
        ("touched", C.c_int64),
        ("ms_total", C.c_double),
        ("ms_sod_kernel", C.c_double),
        ("sod_launches", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("ms_sched", C.c_double),
        ("ms_prep", C.c_double),
        ("ms_refine", C.c_double),
        ("ms_select", C.c_double),
        ("ms_cross", C.c_double),
        ("ncandidates", C.c_int64),
        ("refine_pairs", C.c_int64),
        ("cross_touch", C.c_int64),
        ("refine_slots", C.c_int64),
        ("ms_setup", C.c_double),
        ("ms_output", C.c_double),
        ("ms_learn", C.c_double),
        ("bracket_hits", C.c_int64),
        ("bracket_seeds", C.c_int64),
        ("cross_balls", C.c_int64),
        ("cross_records", C.c_int64),
        ("ms_refine_bound", C.c_double),
        ("refine_items", C.c_int64),
        ("refine_pruned", C.c_int64),
        ("ms_tail", C.c_double),
        ("tail_rounds", C.c_int64),
        ("tail_touch", C.c_int64),
        ("cross_members", C.c_int64),
        ("tail_members", C.c_int64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [("warp_cross_min_ready", C.c_int32), ("bound_min_cand", C.c_int32), ("tail_max_ready", C.c_int32),
                ("tail_max_cand", C.c_int32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class FofParams(C.Structure):
    _fields_ = [("percolation", C.c_float), ("reserved", C.c_int32), ("nres", C.c_int64), ("mmin", C.c_int64)]


class FofStats(C.Structure):
    _fields_ = [
        ("nhalo", C.c_int64),
        ("nmember", C.c_int64),
        ("ngroups", C.c_int64),
        ("fine_cells", C.c_int64),
        ("pair_tests", C.c_int64),
        ("cell_pairs", C.c_int64),
        ("ms_total", C.c_double),
        ("ms_sort", C.c_double),
        ("ms_link", C.c_double),
        ("ms_label", C.c_double),
        ("ms_props", C.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class FofTable(C.Structure):
    _fields_ = [
        ("halo_id", C.c_void_p),
        ("halo_mass", C.c_void_p),
        ("halo_com", C.c_void_p),
        ("halo_vel", C.c_void_p),
        ("halo_radius", C.c_void_p),
        ("member_offset", C.c_void_p),
        ("member_index", C.c_void_p),
        ("member_id", C.c_void_p),
    ]


PROPS_NBIN1 = 100
PROPS_NBIN2 = 30
PROPS_FROM_SOD = 0
PROPS_FROM_FOF = 1


class PropsParams(C.Structure):
    _fields_ = [
        ("unit_l", C.c_double),
        ("unit_d", C.c_double),
        ("unit_t", C.c_double),
        ("aexp", C.c_double),
        ("h0", C.c_double),
        ("hz", C.c_double),
        ("delta_vir", C.c_double),
        ("levelmin", C.c_int32),
        ("center_on_mass", C.c_int32),
        ("periodic", C.c_int32),
        ("source", C.c_int32),
        ("epot_threshold", C.c_int32),
        ("reserved", C.c_int32),
    ]


class PropsStats(C.Structure):
    _fields_ = [("nhalo", C.c_int64), ("nmember", C.c_int64), ("potential_items", C.c_int64),
                ("ms_total", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


# (field, values per halo, numpy dtype) in psod_props_table order
PROPS_FIELDS = [
    ("npart", 1, "int64"), ("mvir", 1, "float64"), ("rvir", 1, "float64"), ("rvircom", 1, "float64"),
    ("vvir", 1, "float64"), ("com", 3, "float32"), ("comv", 3, "float32"), ("rmax", 1, "float32"),
    ("vmax", 1, "float32"), ("dispx", 1, "float32"), ("dispv", 1, "float32"), ("ekin", 1, "float32"),
    ("epot", 1, "float32"), ("lambda", 3, "float32"), ("lambda_prime", 3, "float32"), ("eig_val", 3, "float32"),
    ("eig_vec", 3, "float32"), ("cos_alpha", 1, "float64"), ("center_pot", 3, "float32"), ("circ", 4, "float32"),
    ("delta_vals", 2, "float32"), ("dens", PROPS_NBIN1, "float32"), ("dens_int", PROPS_NBIN1, "float32"),
    ("vcirc", PROPS_NBIN1, "float32"), ("dens178", PROPS_NBIN2, "float32"), ("dens_int178", PROPS_NBIN2, "float32"),
]


class PropsTable(C.Structure):
    _fields_ = [(f, C.c_void_p) for f, _, _ in PROPS_FIELDS]


EXPORTS = [
    "psod_abi_version",
    "psod_status_string",
    "psod_params_default",
    "psod_ctx_create",
    "psod_ctx_destroy",
    "psod_set_stream",
    "psod_load_particles",
    "psod_cic",
    "psod_cicm1",
    "psod_tri_cic",
    "psod_spherover",
    "psod_run",
    "psod_halo_count",
    "psod_get_halos",
    "psod_last_error",
    "psod_cic_rho_static",
    "psod_learn_collect",
    "psod_learn_samples",
    "psod_learn_train",
    "psod_learn_get_model",
    "psod_learn_set_model",
    "psod_learn_set_margin",
    "psod_learn_forward",
    "psod_learn_gradient",
    "psod_write_masst",
    "psod_write_strct",
    "psod_read_cube_zone",
    "psod_select_zone",
    "psod_fof",
    "psod_fof_halo_count",
    "psod_fof_get_halos",
    "psod_halo_properties",
    "psod_props_get",
    "psod_learn_set_features",
    "psod_fof_release",
    "psod_get_tuning",
    "psod_set_tuning",
    "psod_autotune",
]

LEARN_FEATURES = 10
LEARN_PARAMS = 5768
LEARN_MODEL_FLOATS = 5804


class TrainParams(C.Structure):
    _fields_ = [
        ("epochs", C.c_int32),
        ("batch", C.c_int32),
        ("lr", C.c_float),
        ("beta1", C.c_float),
        ("beta2", C.c_float),
        ("eps", C.c_float),
        ("seed", C.c_uint64),
    ]

_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load the in-tree libpsod.so (building it first if asked and needed)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if build_if_missing and not os.path.exists(path):
        _build.build()
    if not os.path.exists(path):
        raise RuntimeError(f"libpsod.so not built at {path}: run psod_b200/build.py")
    L = C.CDLL(path)
    P = C.POINTER
    vp = C.c_void_p
    L.psod_abi_version.restype = C.c_int
    L.psod_status_string.restype = C.c_char_p
    L.psod_status_string.argtypes = [C.c_int]
    L.psod_params_default.argtypes = [P(Params)]
    L.psod_params_default.restype = None
    L.psod_ctx_create.argtypes = [P(Params), P(vp)]
    L.psod_ctx_destroy.argtypes = [vp]
    L.psod_set_stream.argtypes = [vp, vp]
    L.psod_load_particles.argtypes = [vp, C.c_int64, vp, vp, vp, C.c_int64]
    L.psod_cic.argtypes = [vp, vp]
    L.psod_cicm1.argtypes = [vp, vp]
    L.psod_tri_cic.argtypes = [vp, vp, P(C.c_int64)]
    L.psod_spherover.argtypes = [vp, P(RunStats)]
    L.psod_run.argtypes = [vp, P(RunStats)]
    L.psod_halo_count.argtypes = [vp, P(C.c_int64), P(C.c_int64)]
    L.psod_get_halos.argtypes = [vp, P(HaloTable)]
    L.psod_write_masst.argtypes = [C.c_char_p, P(HaloTable), C.c_int64]
    L.psod_write_strct.argtypes = [C.c_char_p, P(HaloTable), C.c_int64, C.c_int64, vp, vp, vp, vp, vp]
    L.psod_read_cube_zone.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int64,
                                      P(C.c_int64), vp, vp, vp]
    L.psod_select_zone.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, C.c_int64, vp, P(C.c_int64)]
    L.psod_fof.argtypes = [vp, P(FofParams), P(FofStats)]
    L.psod_fof_halo_count.argtypes = [vp, P(C.c_int64), P(C.c_int64)]
    L.psod_fof_get_halos.argtypes = [vp, P(FofTable)]
    L.psod_learn_set_features.argtypes = [vp, C.c_int32]
    L.psod_fof_release.argtypes = [vp]
    L.psod_get_tuning.argtypes = [vp, P(Tuning)]
    L.psod_set_tuning.argtypes = [vp, P(Tuning)]
    L.psod_autotune.argtypes = [vp, P(Tuning), P(C.c_double), P(C.c_int32)]
    L.psod_halo_properties.argtypes = [vp, P(PropsParams), P(PropsStats)]
    L.psod_props_get.argtypes = [vp, P(PropsTable)]
    L.psod_last_error.argtypes = [vp]
    L.psod_cic_rho_static.argtypes = [C.c_int64, vp, C.c_int32, C.c_int64, C.c_int32, vp, vp, vp]
    L.psod_learn_collect.argtypes = [vp, C.c_int64]
    L.psod_learn_samples.argtypes = [vp, P(C.c_int64), vp, vp]
    L.psod_learn_train.argtypes = [vp, P(TrainParams), vp]
    L.psod_learn_get_model.argtypes = [vp, vp, C.c_int64]
    L.psod_learn_set_model.argtypes = [vp, vp, C.c_int64]
    L.psod_learn_set_margin.argtypes = [vp, C.c_float]
    L.psod_learn_forward.argtypes = [vp, C.c_int64, vp, vp]
    L.psod_learn_gradient.argtypes = [vp, C.c_int64, vp, vp, vp, vp]
    L.psod_last_error.restype = C.c_char_p
    for name in EXPORTS:
        L[name].restype = L[name].restype if name in ("psod_status_string", "psod_last_error", "psod_params_default") else C.c_int
    _lib = L
    return L


def default_params(nx: int, **kw) -> Params:
    p = Params()
    load().psod_params_default(C.byref(p))
    p.nx = nx
    extra = kw.pop("delta_extra", ())
    for k, v in kw.items():
        setattr(p, k, v)
    p.ndelta_extra = len(extra)
    for i, d in enumerate(extra):
        p.delta_extra[i] = d
    return p
