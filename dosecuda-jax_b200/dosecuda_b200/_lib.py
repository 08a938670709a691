"""ctypes binding of libpb_b200.so (declared in include/pb_b200.h).

The shared library is built in-tree by ``make -C dosecuda-jax_b200/csrc``
(or ``__graft_entry__.build()``).  Importing this module loads it; a missing
library raises ImportError -- there is no CPU fallback for the dose path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpb_b200.so")

PB_OK = 0
PB_ERR_INVALID = 1
PB_ERR_CUDA = 2
PB_ERR_NOMEM = 3
PB_ERR_RAY_CAP = 4
PB_ERR_UNSUPPORTED = 5

PB_MAX_BEAMS = 16
PB_MAX_LUT_LEN = 512
PB_MAX_CURVE = 64
PB_SPOT_GEO_FLOATS = 8
PB_NOALLOC_MAX_WET_FLOATS = 8 * 1024 * 1024


class PbError(RuntimeError):
    """A non-zero PbStatus from the native library."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class PbGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("spacing", ctypes.c_float)]


class PbBeamGeom(ctypes.Structure):
    _fields_ = [("iso", ctypes.c_float * 3), ("src", ctypes.c_float * 3),
                ("singa", ctypes.c_float), ("cosga", ctypes.c_float),
                ("sinta", ctypes.c_float), ("costa", ctypes.c_float),
                ("vsadx", ctypes.c_float), ("vsady", ctypes.c_float)]


class PbSpot(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("mu", ctypes.c_float),
                ("energy_id", ctypes.c_int)]


class PbLayer(ctypes.Structure):
    _fields_ = [("spot_start", ctypes.c_int), ("n_spots", ctypes.c_int),
                ("energy_id", ctypes.c_int), ("r80", ctypes.c_float),
                ("energy", ctypes.c_float),
                ("sx0", ctypes.c_float), ("sx1", ctypes.c_float),
                ("sy0", ctypes.c_float), ("sy1", ctypes.c_float),
                ("sh_max", ctypes.c_float), ("mcs_max", ctypes.c_float),
                ("bound_ok", ctypes.c_int)]


class PbBeam(ctypes.Structure):
    _fields_ = [("geom", PbBeamGeom),
                ("layer_start", ctypes.c_int), ("n_layers", ctypes.c_int),
                ("spot_start", ctypes.c_int), ("n_spots", ctypes.c_int),
                ("dvp_dev", ctypes.c_void_p), ("depths_dev", ctypes.c_void_p),
                ("sigmas_dev", ctypes.c_void_p), ("idds_dev", ctypes.c_void_p),
                ("n_energies", ctypes.c_int), ("lut_len", ctypes.c_int),
                ("dvp_len", ctypes.c_int)]


class PbBatchPlan(ctypes.Structure):
    _fields_ = [("grid", PbGrid), ("n_beams", ctypes.c_int),
                ("beams", PbBeam * PB_MAX_BEAMS),
                ("rlsp_dev", ctypes.c_void_p), ("tex", ctypes.c_uint64),
                ("raw_work_dev", ctypes.c_void_p), ("wet_dev", ctypes.c_void_p),
                ("layers_dev", ctypes.c_void_p), ("spot_geo_dev", ctypes.c_void_p),
                ("mu_dev", ctypes.c_void_p), ("scale", ctypes.c_float),
                ("dose_dev", ctypes.c_void_p)]


class PbBatchInfo(ctypes.Structure):
    _fields_ = [("n_bricks", ctypes.c_longlong), ("n_tiles", ctypes.c_longlong),
                ("n_wet_items", ctypes.c_int), ("n_plans", ctypes.c_int)]


PB_BATCH_WET = 1
PB_BATCH_DOSE = 2

# numpy views of the structs (same layout) for bulk host arrays
SPOT_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("mu", "<f4"), ("energy_id", "<i4")])
LAYER_DTYPE = np.dtype([("spot_start", "<i4"), ("n_spots", "<i4"), ("energy_id", "<i4"),
                        ("r80", "<f4"), ("energy", "<f4"),
                        ("sx0", "<f4"), ("sx1", "<f4"), ("sy0", "<f4"), ("sy1", "<f4"),
                        ("sh_max", "<f4"), ("mcs_max", "<f4"), ("bound_ok", "<i4")])

# Every entry point the header declares, with its argument types.
_VP = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double
_I64 = ctypes.c_int64
_SIGS = {
    "pb_last_error": (ctypes.c_char_p, []),
    "pb_version": (ctypes.c_char_p, []),
    "pb_beam_setup": (_I, [_D, _D, _D, _D, _VP, _VP, ctypes.POINTER(PbBeamGeom)]),
    "pb_build_layers": (_I, [_VP, _I, _VP, _I, _I, _VP, _VP, ctypes.POINTER(_I), _VP]),
    "pb_spot_geometry": (_I, [_VP, _I, _F, _F, _VP]),
    "pb_rlsp_from_hu": (_I, [_VP, _I64, _VP, _VP, _I, _VP, _VP]),
    "pb_texture_create": (_I, [_VP, ctypes.POINTER(PbGrid), ctypes.POINTER(ctypes.c_uint64), _VP]),
    "pb_cells_create": (_I, [_VP, ctypes.POINTER(PbGrid), ctypes.POINTER(ctypes.c_uint64), _VP]),
    "pb_texture_update": (_I, [ctypes.c_uint64, _VP, _VP]),
    "pb_texture_destroy": (_I, [ctypes.c_uint64]),
    "pb_wet": (_I, [_VP, ctypes.c_uint64, ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP]),
    "pb_wet_noalloc": (_I, [_VP, ctypes.c_uint64, ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP]),
    "pb_smooth_table": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _I, _VP, _VP, _VP, _VP]),
    "pb_smooth_dirs": (_I, [_VP, _VP]),
    "pb_dose": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP, _F, _VP, _VP, _VP]),
    "pb_dose_adjoint": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP, _F, _VP,
                             _VP]),
    "pb_dose_variant_count": (_I, []),
    "pb_dose_variant_default": (_I, []),
    "pb_dose_adjoint_variant": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP, _F,
                                     _VP, _I, _VP]),
    "pb_dose_variant_name": (ctypes.c_char_p, [_I]),
    "pb_dose_variant": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP, _F, _VP, _I,
                             _VP]),
    "pb_batch_work_size": (ctypes.c_size_t, [_I]),
    "pb_batch_setup": (_I, [_VP, _I, _VP, ctypes.POINTER(PbBatchInfo), _VP]),
    "pb_batch_run": (_I, [ctypes.POINTER(PbBatchInfo), _VP, _I, _I, _I, _VP, _VP]),
    "pb_objective_work_size": (ctypes.c_size_t, []),
    "pb_objective": (_I, [_VP, _VP, _VP, _I64, _VP, _VP, _VP, _VP]),
    "pb_count_pairs": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP]),
    "pb_layer_bounds": (_I, [_VP, _I, _VP, _VP, _VP]),
    "pb_dose_adjoint_positions": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP, _VP,
                                       _F, _VP, _VP, _VP, _VP]),
    "pb_count_evaluated": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP, _VP]),
    "pb_tile_order_count": (ctypes.c_longlong, [ctypes.POINTER(PbGrid)]),
    "pb_tile_order_tile": (_I, [ctypes.POINTER(ctypes.c_int)]),
    "pb_tile_order_work_size": (ctypes.c_size_t, [ctypes.POINTER(PbGrid)]),
    "pb_tile_order": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP, _VP]),
    "pb_dose_ordered": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP, ctypes.c_float,
                             _VP, _VP, _VP, _VP]),
    "pb_dose_adjoint_ordered": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP,
                                     ctypes.c_float, _VP, _VP, _VP]),
    "pb_count_evaluated_adjoint": (_I, [ctypes.POINTER(PbGrid), _VP, _I, _VP, _VP, _VP, _VP,
                                        ctypes.c_float, _VP, _VP]),
    "pb_measure_ex2_rate": (_I, [ctypes.POINTER(ctypes.c_double), _VP]),
    "pb_host_register": (_I, [_VP, ctypes.c_size_t]),
    "pb_host_unregister": (_I, [_VP]),
    "pb_proton_raytrace_host": (_I, [_I, _D, _D, _VP, _VP, _F, _VP, _VP, _D, _D, _VP]),
    "pb_proton_spot_host": (_I, [_I, _D, _D, _VP, _VP, _VP, _VP, _I, _I, _I, _VP, _VP, _F,
                                 _VP, _VP, _D, _D, _VP, _I, _VP]),
}

EXPORTED = tuple(_SIGS)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C dosecuda-jax_b200/csrc` "
            "(the proton dose path has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    msg = lib.pb_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str = "") -> None:
    """Raise PbError for a non-zero PbStatus."""
    if status != PB_OK:
        text = last_error()
        raise PbError(status, f"{what}: {text}" if what else text)


def ptr(a) -> ctypes.c_void_p:
    """Address of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return ctypes.c_void_p(0)
    if isinstance(a, np.ndarray):
        return ctypes.c_void_p(a.ctypes.data)
    return ctypes.c_void_p(a.data_ptr())


def beam_setup(gantry_deg: float, couch_deg: float, vsadx: float, vsady: float,
               iso, origin) -> PbBeamGeom:
    iso = np.ascontiguousarray(np.asarray(iso, dtype=np.float32).reshape(3))
    origin = np.ascontiguousarray(np.asarray(origin, dtype=np.float32).reshape(3))
    g = PbBeamGeom()
    check(lib.pb_beam_setup(float(gantry_deg), float(couch_deg), float(vsadx), float(vsady),
                            ptr(iso), ptr(origin), ctypes.byref(g)), "pb_beam_setup")
    return g


def smooth_table(shape, spacing: float, geoms, beam: int = 0):
    """The smoothing sample table of one beam, as the WET pass builds it:
    (off [6, 9], hh [6, 9, 3], tmask [6], margin [3]); see pb_smooth_table."""
    nz, ny, nx = shape
    grid = PbGrid(int(nx), int(ny), int(nz), float(spacing))
    arr = (PbBeamGeom * len(geoms))(*geoms)
    off = np.zeros((6, 9), np.int32)
    hh = np.zeros((6, 9, 3), np.float32)
    tmask = np.zeros(6, np.uint32)
    margin = np.zeros(3, np.int32)
    check(lib.pb_smooth_table(ctypes.byref(grid), ctypes.cast(arr, ctypes.c_void_p), len(geoms),
                              int(beam), ptr(off), ptr(hh), ptr(tmask), ptr(margin)),
          "pb_smooth_table")
    return off, hh, tmask, margin


def smooth_dirs():
    """(cos, sin) of the six smoothing directions as the kernels form them
    on the current device (pb_smooth_dirs)."""
    c = np.zeros(6, np.float32)
    s = np.zeros(6, np.float32)
    check(lib.pb_smooth_dirs(ptr(c), ptr(s)), "pb_smooth_dirs")
    return c, s


def build_layers(spot_list: np.ndarray, dvp: np.ndarray):
    """Sorted spots (structured array), layers (structured array), perm."""
    spot_list = np.ascontiguousarray(spot_list, dtype=np.float32).reshape(-1, 4)
    dvp = np.ascontiguousarray(dvp, dtype=np.float32)
    n = spot_list.shape[0]
    n_e, dvp_len = dvp.shape
    spots = np.zeros(n, dtype=SPOT_DTYPE)
    layers = np.zeros(n_e, dtype=LAYER_DTYPE)
    perm = np.zeros(n, dtype=np.int32)
    nl = ctypes.c_int(0)
    check(lib.pb_build_layers(ptr(spot_list), n, ptr(dvp), dvp_len, n_e, ptr(spots),
                              ptr(layers), ctypes.byref(nl), ptr(perm)), "pb_build_layers")
    return spots, layers[: nl.value].copy(), perm


def spot_geometry(spots: np.ndarray, vsadx: float, vsady: float) -> np.ndarray:
    geo = np.zeros((len(spots), PB_SPOT_GEO_FLOATS), dtype=np.float32)
    check(lib.pb_spot_geometry(ptr(spots), len(spots), float(vsadx), float(vsady), ptr(geo)),
          "pb_spot_geometry")
    return geo
