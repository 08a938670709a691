"""Minimal NIfTI-1 writer/reader for 3-D scalar volumes.

Stands in for SimpleITK's NIfTI image I/O behind DoseGrid.writeCTNIFTI
(DoseCUDA/plan.py:214-224).  Volumes are numpy arrays in C order
(nz, ny, nx); the file stores dim = (3, nx, ny, nz), x fastest.  As an ITK
writer does, the patient (LPS) frame is stored as RAS: the qform and sform
are diag(-sx, -sy, sz) with offsets (-ox, -oy, oz), a 180 degree turn about
z (quaternion b = c = 0, d = 1, qfac 1), both with code 1 (scanner frame).
Files ending in .gz are gzip-compressed.
"""
from __future__ import annotations

import gzip
import struct

import numpy as np

_DT = {np.dtype(np.float32): (16, 32), np.dtype(np.float64): (64, 64),
       np.dtype(np.int16): (4, 16), np.dtype(np.uint8): (2, 8), np.dtype(np.int32): (8, 32)}
_DT_BACK = {code: np.dtype(dt) for dt, (code, _) in _DT.items()}
HEADER_SIZE = 348
VOX_OFFSET = 352


def header(shape, dtype, origin, spacing) -> bytes:
    nz, ny, nx = (int(v) for v in shape)
    code, bitpix = _DT[np.dtype(dtype)]
    sx, sy, sz = (float(v) for v in np.asarray(spacing, np.float64).reshape(3))
    ox, oy, oz = (float(v) for v in np.asarray(origin, np.float64).reshape(3))
    h = bytearray(HEADER_SIZE)
    struct.pack_into("<i", h, 0, HEADER_SIZE)                       # sizeof_hdr
    struct.pack_into("<8h", h, 40, 3, nx, ny, nz, 1, 1, 1, 1)       # dim
    struct.pack_into("<hh", h, 70, code, bitpix)                     # datatype, bitpix
    struct.pack_into("<8f", h, 76, 1.0, sx, sy, sz, 0.0, 0.0, 0.0, 0.0)  # pixdim (qfac 1)
    struct.pack_into("<f", h, 108, float(VOX_OFFSET))                # vox_offset
    struct.pack_into("<ff", h, 112, 0.0, 0.0)                        # scl_slope, scl_inter
    struct.pack_into("<B", h, 123, 2)                                # xyzt_units: mm
    struct.pack_into("<hh", h, 252, 1, 1)                            # qform_code, sform_code
    # quatern b, c, d and the offsets
    struct.pack_into("<6f", h, 256, 0.0, 0.0, 1.0, -ox, -oy, oz)
    struct.pack_into("<4f", h, 280, -sx, 0.0, 0.0, -ox)              # srow_x
    struct.pack_into("<4f", h, 296, 0.0, -sy, 0.0, -oy)              # srow_y
    struct.pack_into("<4f", h, 312, 0.0, 0.0, sz, oz)                # srow_z
    h[344:348] = b"n+1\x00"                                          # magic
    return bytes(h)


def write(path: str, volume: np.ndarray, origin, spacing) -> None:
    vol = np.asarray(volume)
    if vol.ndim != 3:
        raise ValueError("NIfTI writer takes a 3-D volume")
    if vol.dtype not in _DT:
        vol = vol.astype(np.float32)
    vol = np.ascontiguousarray(vol.astype(vol.dtype.newbyteorder("<")))
    data = header(vol.shape, vol.dtype, origin, spacing) + b"\x00" * 4 + vol.tobytes()
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "wb") as f:
        f.write(data)


def read(path: str):
    """Return (volume (nz, ny, nx), origin (3,), spacing (3,)) of a file this
    module wrote (LPS origin from the sform)."""
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rb") as f:
        data = f.read()
    if struct.unpack_from("<i", data, 0)[0] != HEADER_SIZE or data[344:347] != b"n+1":
        raise ValueError(f"{path}: not a single-file NIfTI-1 image")
    dim = struct.unpack_from("<8h", data, 40)
    code = struct.unpack_from("<h", data, 70)[0]
    pixdim = struct.unpack_from("<8f", data, 76)
    off = int(struct.unpack_from("<f", data, 108)[0])
    nx, ny, nz = dim[1], dim[2], dim[3]
    dt = _DT_BACK[code]
    vol = np.frombuffer(data, dtype=dt.newbyteorder("<"), count=nx * ny * nz,
                        offset=off).reshape(nz, ny, nx)
    sx = struct.unpack_from("<4f", data, 280)
    sy = struct.unpack_from("<4f", data, 296)
    sz = struct.unpack_from("<4f", data, 312)
    origin = np.array([-sx[3], -sy[3], sz[3]], np.float64)
    return vol.astype(dt.newbyteorder("=")), origin, np.array(pixdim[1:4], np.float64)
