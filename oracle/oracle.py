"""Python wrapper of the CPU oracle (liboracle.so / libport32.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference legs may
import this module.  The product (dosecuda_b200) never imports it.

The C restatement is oracle/pb_oracle.c (see its header for the reference
file:line map).  HU -> RLSP is numpy.interp, the reference's own call
(DoseCUDA/plan_impt.py:158-168).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class OBeam(ctypes.Structure):
    _fields_ = [("iso", ctypes.c_float * 3), ("src", ctypes.c_float * 3),
                ("singa", ctypes.c_float), ("cosga", ctypes.c_float),
                ("sinta", ctypes.c_float), ("costa", ctypes.c_float),
                ("vsadx", ctypes.c_float), ("vsady", ctypes.c_float)]


class OGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("s", ctypes.c_float)]


class OModel(ctypes.Structure):
    _fields_ = [("dvp", ctypes.c_void_p), ("depths", ctypes.c_void_p),
                ("sigmas", ctypes.c_void_p), ("idds", ctypes.c_void_p),
                ("dvp_len", ctypes.c_int), ("lut_len", ctypes.c_int),
                ("n_energies", ctypes.c_int)]


SPOT = np.dtype([("x", "<f4"), ("y", "<f4"), ("mu", "<f4"), ("energy_id", "<i4")])
LAYER = np.dtype([("spot_start", "<i4"), ("n_spots", "<i4"), ("energy_id", "<i4"),
                  ("r80", "<f4"), ("energy", "<f4")])

_LIBS = {}


def _p(a):
    return ctypes.c_void_p(0) if a is None else ctypes.c_void_p(a.ctypes.data)


def load(port32: bool = False):
    """Load liboracle.so (FP64) or libport32.so (FP32, timed baseline),
    building them with `make -C oracle` if absent."""
    name = "libport32.so" if port32 else "liboracle.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        subprocess.run(["make", "-C", HERE, name], check=True, capture_output=True)
    lib = ctypes.CDLL(path)
    real = ctypes.c_float if port32 else ctypes.c_double
    vp, i, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
    lib.ob_beam_setup.argtypes = [ctypes.c_double] * 4 + [vp, vp, ctypes.POINTER(OBeam)]
    lib.ob_smooth_dirs.argtypes = [vp, vp]
    lib.ob_set_smooth_dirs.argtypes = [vp, vp]
    lib.ob_set_fuse.argtypes = [vp]
    lib.ob_raytrace.argtypes = [vp, ctypes.POINTER(OGrid), ctypes.POINTER(OBeam), vp, i64, vp]
    lib.ob_raytrace.restype = i
    lib.ob_smooth.argtypes = [vp, ctypes.POINTER(OGrid), ctypes.POINTER(OBeam), vp, i64, vp]
    lib.ob_smooth_f32.argtypes = [vp, ctypes.POINTER(OGrid), ctypes.POINTER(OBeam), vp]
    lib.ob_smooth_choices.argtypes = [ctypes.POINTER(OGrid), ctypes.POINTER(OBeam), vp]
    lib.ob_build_layers.argtypes = [vp, i, vp, i, i, vp, vp]
    lib.ob_build_layers.restype = i
    lib.ob_dose.argtypes = [vp, ctypes.POINTER(OGrid), ctypes.POINTER(OBeam),
                            ctypes.POINTER(OModel), vp, vp, i, vp, i64, vp]
    lib.ob_adjoint.argtypes = [vp, ctypes.POINTER(OGrid), ctypes.POINTER(OBeam),
                               ctypes.POINTER(OModel), vp, vp, i, vp, vp]
    lib.ob_count_pairs.argtypes = [vp, i64, vp, i]
    lib.ob_count_pairs.restype = i64
    lib.ob_real_size.restype = i
    lib._real = np.float32 if port32 else np.float64
    lib._creal = real
    _LIBS[name] = lib
    return lib


def beam_setup(gantry, couch, vsadx, vsady, iso, origin, port32=False) -> OBeam:
    lib = load(port32)
    b = OBeam()
    iso = np.ascontiguousarray(np.asarray(iso, np.float32).reshape(3))
    origin = np.ascontiguousarray(np.asarray(origin, np.float32).reshape(3))
    lib.ob_beam_setup(float(gantry), float(couch), float(vsadx), float(vsady), _p(iso),
                      _p(origin), ctypes.byref(b))
    return b


def set_smooth_dirs(c=None, s=None):
    """Use these smoothing directions (cos, sin of i*pi/3, FP32) in every
    smoothing call, as the reference's device sincosf gives them; None goes
    back to the C library's values."""
    for port32 in (False, True):
        lib = load(port32)
        if c is None:
            lib.ob_set_smooth_dirs(None, None)
        else:
            cc = np.ascontiguousarray(c, np.float32)
            ss = np.ascontiguousarray(s, np.float32)
            lib.ob_set_smooth_dirs(_p(cc), _p(ss))


def set_fuse(modes=None):
    """Fused multiply-adds in the FP32 rotations and smoothing samples (see
    ob_set_fuse): nine modes, or None for the reference's own pattern."""
    for port32 in (False, True):
        lib = load(port32)
        if modes is None:
            lib.ob_set_fuse(None)
        else:
            m = np.ascontiguousarray(modes, np.int32)
            assert m.shape == (9,)
            lib.ob_set_fuse(_p(m))


def smooth_dirs():
    lib = load()
    c = np.zeros(6, np.float32)
    s = np.zeros(6, np.float32)
    lib.ob_smooth_dirs(_p(c), _p(s))
    return c, s


def _grid(shape, spacing) -> OGrid:
    nz, ny, nx = shape
    return OGrid(int(nx), int(ny), int(nz), float(np.float32(spacing)))


def rlsp_from_hu(hu, curve_hu, curve_rlsp):
    return np.array(np.interp(hu, curve_hu, curve_rlsp), dtype=np.single)


def raytrace(rlsp, spacing, beam: OBeam, idx=None, port32=False):
    """Raw WET (cm) per voxel (or per index in idx)."""
    lib = load(port32)
    rlsp = np.ascontiguousarray(rlsp, np.float32)
    n = rlsp.size if idx is None else len(idx)
    idx = None if idx is None else np.ascontiguousarray(idx, np.int64)
    out = np.zeros(n, lib._real)
    err = lib.ob_raytrace(_p(rlsp), ctypes.byref(_grid(rlsp.shape, spacing)), ctypes.byref(beam),
                          _p(idx), 0 if idx is None else len(idx), _p(out))
    if err:
        raise RuntimeError("oracle ray reached its step cap")
    return out if idx is not None else out.reshape(rlsp.shape)


def smooth(raw_f32, spacing, beam: OBeam, idx=None, port32=False):
    lib = load(port32)
    raw = np.ascontiguousarray(raw_f32, np.float32)
    n = raw.size if idx is None else len(idx)
    idx = None if idx is None else np.ascontiguousarray(idx, np.int64)
    out = np.zeros(n, lib._real)
    lib.ob_smooth(_p(raw), ctypes.byref(_grid(raw.shape, spacing)), ctypes.byref(beam), _p(idx),
                  0 if idx is None else len(idx), _p(out))
    return out if idx is not None else out.reshape(raw.shape)


def smooth_f32(raw_f32, spacing, beam: OBeam):
    """The smoothing with the reference's FP32 sum and quotient: equal bit
    for bit to a kernel that picks the same sample voxels."""
    lib = load()
    raw = np.ascontiguousarray(raw_f32, np.float32)
    out = np.zeros(raw.shape, np.float32)
    lib.ob_smooth_f32(_p(raw), ctypes.byref(_grid(raw.shape, spacing)), ctypes.byref(beam),
                      _p(out))
    return out


def smooth_choices(shape, spacing, beam: OBeam):
    """Index (i, j, k) the reference picks for every smoothing sample of
    every voxel: int32 [nz, ny, nx, 6 directions, 9 radii, 3 axes]."""
    lib = load()
    out = np.zeros(tuple(shape) + (6, 9, 3), np.int32)
    lib.ob_smooth_choices(ctypes.byref(_grid(shape, spacing)), ctypes.byref(beam), _p(out))
    return out


def build_layers(spot_list, dvp):
    lib = load()
    sl = np.ascontiguousarray(np.asarray(spot_list, np.float32).reshape(-1, 4))
    dvp = np.ascontiguousarray(dvp, np.float32)
    spots = np.zeros(len(sl), SPOT)
    layers = np.zeros(dvp.shape[0], LAYER)
    nl = lib.ob_build_layers(_p(sl), len(sl), _p(dvp), dvp.shape[1], dvp.shape[0], _p(spots),
                             _p(layers))
    return spots, layers[:nl].copy()


class Model:
    """Keeps the model arrays alive while the oracle holds pointers."""

    def __init__(self, model):
        self.dvp = np.ascontiguousarray(model.divergence_params, np.float32)
        self.dep = np.ascontiguousarray(model.lut_depths, np.float32)
        self.sig = np.ascontiguousarray(model.lut_sigmas, np.float32)
        self.idd = np.ascontiguousarray(model.lut_idds, np.float32)
        self.c = OModel(self.dvp.ctypes.data, self.dep.ctypes.data, self.sig.ctypes.data,
                        self.idd.ctypes.data, self.dvp.shape[1], self.dep.shape[1],
                        self.dvp.shape[0])
        self.vsadx = float(model.VSADX)
        self.vsady = float(model.VSADY)


def dose(wet_cm_f32, spacing, beam: OBeam, model: Model, spots, layers, idx=None,
         port32=False):
    """Beam dose (FP64 in liboracle) at every voxel or at idx."""
    lib = load(port32)
    wet = np.ascontiguousarray(wet_cm_f32, np.float32)
    n = wet.size if idx is None else len(idx)
    idx = None if idx is None else np.ascontiguousarray(idx, np.int64)
    out = np.zeros(n, lib._real)
    spots = np.ascontiguousarray(spots)
    layers = np.ascontiguousarray(layers)
    lib.ob_dose(_p(wet), ctypes.byref(_grid(wet.shape, spacing)), ctypes.byref(beam),
                ctypes.byref(model.c), _p(spots), _p(layers), len(layers), _p(idx),
                0 if idx is None else len(idx), _p(out))
    return out if idx is not None else out.reshape(wet.shape)


def adjoint(wet_cm_f32, spacing, beam: OBeam, model: Model, spots, layers, w):
    """grad[s] = sum_v w[v] K(v, s), sorted spot order, FP64."""
    lib = load()
    wet = np.ascontiguousarray(wet_cm_f32, np.float32)
    w = np.ascontiguousarray(w, np.float64).reshape(-1)
    g = np.zeros(len(spots), np.float64)
    lib.ob_adjoint(_p(wet), ctypes.byref(_grid(wet.shape, spacing)), ctypes.byref(beam),
                   ctypes.byref(model.c), _p(np.ascontiguousarray(spots)),
                   _p(np.ascontiguousarray(layers)), len(layers), _p(w), _p(g))
    return g


def count_pairs(wet_cm_f32, layers):
    lib = load()
    wet = np.ascontiguousarray(wet_cm_f32, np.float32)
    return int(lib.ob_count_pairs(_p(wet), wet.size, _p(np.ascontiguousarray(layers)),
                                  len(layers)))


def plan_forward(hu, origin, spacing, beams, curve, want_raw=False):
    """Oracle version of computeIMPTPlan without n_fractions: returns dict
    with per-beam raw/smoothed WET (float32) and dose (FP64), and the sum.

    beams: list of (gantry, couch, iso, spot_list, model)."""
    rlsp = rlsp_from_hu(hu, *curve)
    out = {"rlsp": rlsp, "wet": [], "raw": [], "beam_dose": [], "layers": [], "spots": []}
    total = np.zeros(rlsp.shape, np.float64)
    for (g, c, iso, sl, model) in beams:
        m = Model(model)
        b = beam_setup(g, c, m.vsadx, m.vsady, iso, origin)
        raw = raytrace(rlsp, spacing, b).astype(np.float32)
        wet = smooth(raw, spacing, b).astype(np.float32)
        spots, layers = build_layers(sl, m.dvp)
        d = dose(wet, spacing, b, m, spots, layers)
        total += d
        out["wet"].append(wet)
        if want_raw:
            out["raw"].append(raw)
        out["beam_dose"].append(d)
        out["layers"].append(layers)
        out["spots"].append(spots)
    out["dose"] = total
    return out
