"""Drop-in for the reference's ``dose_kernels`` CPython module (proton part).

Same two functions, same attribute contract, same error types as
DoseCUDA/dose_kernels/dosemodule.cu:104-201 (proton_raytrace) and
:243-374 (proton_spot), backed by libpb_b200.so's host-buffer entry points
pb_proton_raytrace_host / pb_proton_spot_host:

  proton_raytrace_cuda(model, volume, beam, gpu_id) -> float32 ndarray
      smoothed WET (cm), same shape as volume.voxel_data
  proton_spot_cuda(model, volume, wet_volume, beam, gpu_id) -> float32 ndarray
      dose of the beam for its weights as given (no n_fractions factor)

Attribute rules (dosemodule.cu:23-101): arrays must be numpy float32 of the
stated rank, else ValueError("'<attr>' must be N-dimensional and of type
float."); a missing attribute raises AttributeError; scalars go through the
float protocol.  CUDA failures raise RuntimeError("CUDA error: ...").
Non-contiguous arrays are copied to C order first (the reference reads raw
pointers without a contiguity check).
"""
from __future__ import annotations

import ctypes
import operator

import numpy as np

from . import _lib
from ._lib import PbError, ptr


def _getarray(obj, attr: str, dim: int) -> np.ndarray:
    a = getattr(obj, attr)
    if not (isinstance(a, np.ndarray) and a.ndim == dim and a.dtype == np.float32):
        raise ValueError("'%s' must be %d-dimensional and of type float." % (attr, dim))
    return np.ascontiguousarray(a)


def _getfloat(obj, attr: str) -> float:
    v = getattr(obj, attr)
    if isinstance(v, (str, bytes)):
        raise TypeError("must be real number, not %s" % type(v).__name__)
    if hasattr(v, "__float__"):
        return float(v)
    try:
        return float(operator.index(v))
    except TypeError:
        raise TypeError("must be real number, not %s" % type(v).__name__) from None


def _raise(e: PbError):
    if e.code == _lib.PB_ERR_INVALID:
        raise ValueError(str(e)) from None
    raise RuntimeError("CUDA error: %s" % e) from None


def _call(fn, *args, what=""):
    status = fn(*args)
    if status != _lib.PB_OK:
        _raise(PbError(status, _lib.last_error()))


def proton_raytrace_cuda(model_instance, volume_instance, beam_instance, gpu_id):
    """Compute WET array for proton dose calc."""
    gpu_id = operator.index(gpu_id)
    vsadx = _getfloat(model_instance, "VSADX")
    vsady = _getfloat(model_instance, "VSADY")
    density = _getarray(volume_instance, "voxel_data", 3)
    spacing = _getarray(volume_instance, "spacing", 1)
    origin = _getarray(volume_instance, "origin", 1)
    iso = _getarray(beam_instance, "iso", 1)
    ga = _getfloat(beam_instance, "gantry_angle")
    ta = _getfloat(beam_instance, "couch_angle")
    dims = np.array(density.shape, dtype=np.int64)
    out = np.empty(density.shape, dtype=np.float32)
    _call(_lib.lib.pb_proton_raytrace_host, gpu_id, vsadx, vsady, ptr(density), ptr(dims),
          ctypes.c_float(spacing[0]), ptr(origin), ptr(iso), ga, ta, ptr(out))
    return out


def proton_spot_cuda(model_instance, volume_instance, wet_instance, beam_instance, gpu_id):
    """Compute proton spot dose with PB using pre-calc'd WET array."""
    gpu_id = operator.index(gpu_id)
    vsadx = _getfloat(model_instance, "VSADX")
    vsady = _getfloat(model_instance, "VSADY")
    dvp = _getarray(model_instance, "divergence_params", 2)
    depths = _getarray(model_instance, "lut_depths", 2)
    sigmas = _getarray(model_instance, "lut_sigmas", 2)
    idds = _getarray(model_instance, "lut_idds", 2)
    _getarray(volume_instance, "voxel_data", 3)
    spacing = _getarray(volume_instance, "spacing", 1)
    origin = _getarray(volume_instance, "origin", 1)
    wet = _getarray(wet_instance, "voxel_data", 3)
    iso = _getarray(beam_instance, "iso", 1)
    spots = _getarray(beam_instance, "spot_list", 2)
    ga = _getfloat(beam_instance, "gantry_angle")
    ta = _getfloat(beam_instance, "couch_angle")
    if spots.shape[0] and spots.shape[1] != 4:
        raise ValueError("'spot_list' must have 4 columns (x, y, mu, energy_id).")
    if depths.shape != sigmas.shape or depths.shape != idds.shape or \
            dvp.shape[0] != depths.shape[0] or dvp.shape[1] < 5:
        raise ValueError("beam model tables have inconsistent shapes.")
    dims = np.array(wet.shape, dtype=np.int64)
    out = np.empty(wet.shape, dtype=np.float32)
    _call(_lib.lib.pb_proton_spot_host, gpu_id, vsadx, vsady, ptr(dvp), ptr(depths), ptr(sigmas),
          ptr(idds), depths.shape[0], depths.shape[1], dvp.shape[1], ptr(wet), ptr(dims),
          ctypes.c_float(spacing[0]), ptr(origin), ptr(iso), ga, ta, ptr(spots), spots.shape[0],
          ptr(out))
    return out
