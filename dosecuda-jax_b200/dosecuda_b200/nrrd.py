"""Minimal NRRD reader/writer for 3-D scalar volumes.

Stands in for the SimpleITK image I/O that the reference plan classes use
(DoseCUDA/plan.py:33-41 loadCTNRRD, :173-212 writeDoseNRRD/writeCTNRRD,
plan_impt.py:259-287 writeWETNRRD).  Volumes are numpy arrays in C order
(nz, ny, nx); the file stores sizes as (nx, ny, nz), x fastest, like an
image written by SimpleITK.GetImageFromArray.  Writes raw or gzip encoding;
reads raw and gzip.
"""
from __future__ import annotations

import gzip

import numpy as np

_TYPES = {
    np.dtype(np.float32): "float",
    np.dtype(np.float64): "double",
    np.dtype(np.int16): "short",
    np.dtype(np.uint16): "unsigned short",
    np.dtype(np.int32): "int",
    np.dtype(np.uint8): "unsigned char",
}
_NAMES = {
    "float": np.float32, "double": np.float64, "short": np.int16, "int16": np.int16,
    "signed short": np.int16, "unsigned short": np.uint16, "ushort": np.uint16,
    "uint16": np.uint16, "int": np.int32, "int32": np.int32, "signed int": np.int32,
    "unsigned char": np.uint8, "uchar": np.uint8, "uint8": np.uint8,
}


def write(path: str, volume: np.ndarray, origin, spacing, compress: bool = False) -> None:
    vol = np.asarray(volume)
    if vol.ndim != 3:
        raise ValueError("NRRD writer takes a 3-D volume")
    if vol.dtype not in _TYPES:
        vol = vol.astype(np.float32)
    vol = np.ascontiguousarray(vol.astype(vol.dtype.newbyteorder("<")))
    nz, ny, nx = vol.shape
    sx, sy, sz = (float(v) for v in np.asarray(spacing, dtype=np.float64).reshape(3))
    ox, oy, oz = (float(v) for v in np.asarray(origin, dtype=np.float64).reshape(3))
    header = [
        "NRRD0004",
        f"type: {_TYPES[vol.dtype]}",
        "dimension: 3",
        "space: left-posterior-superior",
        f"sizes: {nx} {ny} {nz}",
        f"space directions: ({sx!r},0,0) (0,{sy!r},0) (0,0,{sz!r})",
        "kinds: domain domain domain",
        "endian: little",
        f"encoding: {'gzip' if compress else 'raw'}",
        f"space origin: ({ox!r},{oy!r},{oz!r})",
    ]
    payload = vol.tobytes()
    if compress:
        payload = gzip.compress(payload)
    with open(path, "wb") as f:
        f.write(("\n".join(header) + "\n\n").encode("ascii"))
        f.write(payload)


def read(path: str):
    """Return (volume (nz, ny, nx), origin (3,), spacing (3,))."""
    with open(path, "rb") as f:
        data = f.read()
    end = data.find(b"\n\n")
    if not data.startswith(b"NRRD") or end < 0:
        raise ValueError(f"{path}: not an NRRD file with an attached payload")
    fields = {}
    for line in data[:end].decode("ascii").splitlines()[1:]:
        if not line or line.startswith("#") or ":" not in line:
            continue
        key, _, val = line.partition(":")
        fields[key.strip().lower()] = val.strip().lstrip("=").strip()
    sizes = [int(v) for v in fields["sizes"].split()]
    if len(sizes) != 3:
        raise ValueError("NRRD reader takes 3-D volumes")
    dtype = np.dtype(_NAMES[fields["type"].lower()])
    if fields.get("endian", "little") == "big":
        dtype = dtype.newbyteorder(">")
    payload = data[end + 2:]
    enc = fields.get("encoding", "raw").lower()
    if enc in ("gzip", "gz"):
        payload = gzip.decompress(payload)
    elif enc != "raw":
        raise ValueError(f"unsupported NRRD encoding {enc!r}")
    nx, ny, nz = sizes
    vol = np.frombuffer(payload, dtype=dtype, count=nx * ny * nz).reshape(nz, ny, nx)
    spacing = np.ones(3)
    if "space directions" in fields:
        vecs = fields["space directions"].replace(")", "").split("(")[1:]
        spacing = np.array([np.linalg.norm([float(c) for c in v.split(",")]) for v in vecs])
    elif "spacings" in fields:
        spacing = np.array([float(v) for v in fields["spacings"].split()])
    origin = np.zeros(3)
    if "space origin" in fields:
        origin = np.array([float(c) for c in fields["space origin"].strip("()").split(",")])
    return vol.astype(dtype.newbyteorder("=")), origin, spacing
