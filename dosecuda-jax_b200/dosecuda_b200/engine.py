"""Device-resident plan state and the calls into libpb_b200.so.

torch provides device memory and the current stream; every computation is a
C-ABI call (include/pb_b200.h) that launches the package's sm_100a kernels.

A ``DevicePlan`` holds, on one GPU, everything the pencil-beam kernels read
for one plan: the grid, per-beam geometry and model tables, the layers and
per-spot geometry in sorted (layer) order, the spot weights and the WET of
every beam.  It exposes the forward dose, the adjoint (spot-weight
gradient) and the dense pair count, so that an optimisation loop keeps all
state on the device (reference host round trips: IMPTClasses.cu:274-340,
plan_impt.py:185-206).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import PbBeam, PbGrid, check, ptr


def _stream(device: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def require_cuda(device) -> torch.device:
    dev = torch.device(device)
    if dev.type != "cuda":
        raise ValueError("the pencil-beam dose path runs on CUDA devices only")
    if not torch.cuda.is_available():
        raise RuntimeError("CUDA error: no CUDA device is available")
    return dev


@dataclass
class ModelTables:
    """One beam model's tables on one device (plan_impt.py:63-149)."""
    dvp: torch.Tensor
    depths: torch.Tensor
    sigmas: torch.Tensor
    idds: torch.Tensor
    n_energies: int
    lut_len: int
    dvp_len: int
    dvp_host: np.ndarray


def model_tables(model, device: torch.device) -> ModelTables:
    """Upload (once per device) the LUTs of an IMPTBeamModel-like object."""
    cache = model.__dict__.setdefault("_pb_device_tables", {})
    key = (device.index, id(model.divergence_params), id(model.lut_depths))
    hit = cache.get(key)
    if hit is not None:
        return hit
    dvp = np.ascontiguousarray(model.divergence_params, dtype=np.float32)
    dep = np.ascontiguousarray(model.lut_depths, dtype=np.float32)
    sig = np.ascontiguousarray(model.lut_sigmas, dtype=np.float32)
    idd = np.ascontiguousarray(model.lut_idds, dtype=np.float32)
    if dvp.ndim != 2 or dvp.shape[1] < 5:
        raise ValueError("divergence_params must be n_energies x 5 (energy, R80, A, B, C)")
    if dep.ndim != 2 or dep.shape != sig.shape or dep.shape != idd.shape:
        raise ValueError("lut_depths / lut_sigmas / lut_idds must share one 2-D shape")
    if dep.shape[0] != dvp.shape[0]:
        raise ValueError("LUT rows and divergence_params rows differ")
    if dep.shape[1] > _lib.PB_MAX_LUT_LEN:
        raise ValueError(f"LUT length {dep.shape[1]} exceeds {_lib.PB_MAX_LUT_LEN}")
    t = ModelTables(
        dvp=torch.from_numpy(dvp).to(device), depths=torch.from_numpy(dep).to(device),
        sigmas=torch.from_numpy(sig).to(device), idds=torch.from_numpy(idd).to(device),
        n_energies=dvp.shape[0], lut_len=dep.shape[1], dvp_len=dvp.shape[1], dvp_host=dvp)
    cache[key] = t
    return t


def rlsp_from_hu(hu: torch.Tensor, curve_hu: np.ndarray, curve_rlsp: np.ndarray,
                 out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """HU -> RLSP on the GPU with numpy.interp semantics (plan_impt.py:158-168)."""
    if hu.dtype != torch.float32 or not hu.is_cuda:
        raise ValueError("hu must be a float32 CUDA tensor")
    hu = hu.contiguous()
    if out is None:
        out = torch.empty_like(hu)
    xh = np.ascontiguousarray(curve_hu, dtype=np.float64)
    yh = np.ascontiguousarray(curve_rlsp, dtype=np.float64)
    check(_lib.lib.pb_rlsp_from_hu(ptr(hu), hu.numel(), ptr(xh), ptr(yh), len(xh), ptr(out),
                                   _stream(hu.device)), "pb_rlsp_from_hu")
    return out


@dataclass
class BeamSpec:
    """What the kernels need from one beam of a plan."""
    gantry_angle: float
    couch_angle: float
    iso: np.ndarray
    spot_list: np.ndarray      # n x 4 float32 (x, y, mu, energy_id)
    model: object              # IMPTBeamModel-like


def grid_of(volume_shape: Sequence[int], spacing: float) -> PbGrid:
    nz, ny, nx = (int(v) for v in volume_shape)
    return PbGrid(nx, ny, nz, float(spacing))


class TexturePool:
    """Texture and cell-record handles kept across the plans of one grid,
    so that repeated dose calls on the same CT refill them instead of
    allocating and freeing them every time (the reference creates and
    destroys its texture on every call, TextureClasses.cu:14-41).  Plans
    that share a pool must run one at a time in stream order on one
    stream: a pooled handle holds the RLSP it was last filled with."""

    def __init__(self):
        self._handles = {}

    def holder(self, device: torch.device, shape, kind: str) -> ctypes.c_uint64:
        key = (device.index, tuple(int(v) for v in shape), kind)
        h = self._handles.get(key)
        if h is None:
            h = ctypes.c_uint64(0)
            self._handles[key] = h
        return h

    def close(self) -> None:
        for (dev, _, _), h in list(self._handles.items()):
            if h.value:
                try:
                    torch.cuda.synchronize(dev)
                    _lib.lib.pb_texture_destroy(h)
                except Exception:
                    pass
                h.value = 0
        self._handles.clear()

    def __del__(self):
        self.close()


def split_order_by_slabs(order: torch.Tensor, dims, tile, n_parts: int):
    """A tile order (a permutation of the raster tile indices, x fastest, for
    a grid of dims = (nx, ny, nz) voxels in tiles of tile = (tx, ty, tz)
    voxels) split into up to n_parts groups of whole z slabs of tiles,
    lowest z first: a list of (order, v0, v1).  Each order keeps the group's
    tiles in their given order and is padded with -1 to the full count; it
    covers exactly voxels v0 <= v < v1 (z varies slowest).  Stream-ordered
    on the order's device."""
    nx, ny, nz = (int(v) for v in dims)
    per_slab = -(-nx // int(tile[0])) * -(-ny // int(tile[1]))
    n_slabs = -(-nz // int(tile[2]))
    n_parts = max(1, min(int(n_parts), n_slabs))
    if n_parts == 1:
        return [(order, 0, nx * ny * nz)]
    # group of slab tz: tz * n_parts // n_slabs (non-decreasing in tz)
    group = (order // per_slab) * n_parts // n_slabs
    ranked = order[torch.sort(group, stable=True).indices]
    pad = torch.full((order.numel(),), -1, dtype=order.dtype, device=order.device)
    parts, t0, z0 = [], 0, 0
    for p in range(n_parts):
        z1 = z0
        while z1 < n_slabs and z1 * n_parts // n_slabs == p:
            z1 += 1
        t1 = t0 + (z1 - z0) * per_slab
        part = torch.cat([ranked[t0:t1], pad[:order.numel() - (t1 - t0)]])
        parts.append((part, nx * ny * min(z0 * int(tile[2]), nz),
                      nx * ny * min(z1 * int(tile[2]), nz)))
        t0, z0 = t1, z1
    return parts


class DevicePlan:
    """A plan prepared on one GPU (see module docstring)."""

    def __init__(self, volume_shape, spacing: float, origin, beams: List[BeamSpec],
                 device="cuda", texture_pool: Optional[TexturePool] = None,
                 defer_spots: bool = False):
        """defer_spots: set up the beam geometry only (enough for the WET);
        load_spots() then sorts the spots into layers and uploads them, for
        instance on another stream while the WET runs."""
        self.device = require_cuda(device)
        if not beams:
            raise ValueError("a plan needs at least one beam")
        if len(beams) > _lib.PB_MAX_BEAMS:
            raise ValueError(f"at most {_lib.PB_MAX_BEAMS} beams per plan")
        self.shape = tuple(int(v) for v in volume_shape)
        self.grid = grid_of(self.shape, spacing)
        self.n_vox = int(np.prod(self.shape))
        self.n_beams = len(beams)
        origin = np.asarray(origin, dtype=np.float32).reshape(3)

        self.geoms = (_lib.PbBeamGeom * self.n_beams)()
        self.tables: List[ModelTables] = []
        for b, bs in enumerate(beams):
            self.tables.append(model_tables(bs.model, self.device))
            self.geoms[b] = _lib.beam_setup(bs.gantry_angle, bs.couch_angle, bs.model.VSADX,
                                            bs.model.VSADY, bs.iso, origin)
        self.wet: Optional[torch.Tensor] = None
        self._status = torch.zeros(1, dtype=torch.int32, device=self.device)
        # texture / cell-record handles: the plan's own, or a pool's
        self._owns_textures = texture_pool is None
        if texture_pool is None:
            self._tex = ctypes.c_uint64(0)
            self._cells = ctypes.c_uint64(0)
        else:
            self._tex = texture_pool.holder(self.device, self.shape, "texture")
            self._cells = texture_pool.holder(self.device, self.shape, "cells")
        self.wet_mode = "texture"
        self._spec = beams
        self._order: Optional[torch.Tensor] = None    # tile order for the current WET
        self._beam_orders: Optional[list] = None      # each beam's own tile order
        self._order_work: Optional[torch.Tensor] = None
        self.spots_loaded = False
        if not defer_spots:
            self.load_spots()

    def load_spots(self) -> None:
        """Spots sorted into energy layers, their geometry, the layer
        records and their culling bounds, on the device (stream-ordered on
        the current stream)."""
        if self.spots_loaded:
            return
        layer_blocks, geo_blocks, mu_blocks, perm_blocks = [], [], [], []
        self.spot_offsets = [0]
        self.layer_offsets = [0]
        self.n_layers: List[int] = []
        for b, bs in enumerate(self._spec):
            t = self.tables[b]
            sl = np.ascontiguousarray(bs.spot_list, dtype=np.float32).reshape(-1, 4)
            spots, layers, perm = _lib.build_layers(sl, t.dvp_host)
            geo = _lib.spot_geometry(spots, self.geoms[b].vsadx, self.geoms[b].vsady)
            layer_blocks.append(layers)
            geo_blocks.append(geo)
            mu_blocks.append(spots["mu"].astype(np.float32))
            perm_blocks.append(perm.astype(np.int64) + self.spot_offsets[-1])
            self.spot_offsets.append(self.spot_offsets[-1] + len(spots))
            self.layer_offsets.append(self.layer_offsets[-1] + len(layers))
            self.n_layers.append(len(layers))
        self.n_spots = self.spot_offsets[-1]
        layers_all = np.concatenate(layer_blocks) if self.layer_offsets[-1] else \
            np.zeros(1, dtype=_lib.LAYER_DTYPE)
        geo_all = np.concatenate(geo_blocks) if self.n_spots else \
            np.zeros((1, _lib.PB_SPOT_GEO_FLOATS), np.float32)
        self.layers_np = layers_all
        self.layers = torch.from_numpy(layers_all.view(np.uint8).copy()).to(self.device)
        self.spot_geo = torch.from_numpy(np.ascontiguousarray(geo_all)).to(self.device)
        # sorted position q holds the spot of plan row perm[q]
        self.perm = torch.from_numpy(np.concatenate(perm_blocks) if self.n_spots
                                     else np.zeros(0, np.int64)).to(self.device)
        mu_sorted = np.concatenate(mu_blocks) if self.n_spots else np.zeros(0, np.float32)
        self.mu_sorted = torch.from_numpy(mu_sorted).to(self.device)
        self.beams = (PbBeam * self.n_beams)()
        for b in range(self.n_beams):
            t = self.tables[b]
            B = self.beams[b]
            B.geom = self.geoms[b]
            B.layer_start = self.layer_offsets[b]
            B.n_layers = self.n_layers[b]
            B.spot_start = self.spot_offsets[b]
            B.n_spots = self.spot_offsets[b + 1] - self.spot_offsets[b]
            B.dvp_dev = t.dvp.data_ptr()
            B.depths_dev = t.depths.data_ptr()
            B.sigmas_dev = t.sigmas.data_ptr()
            B.idds_dev = t.idds.data_ptr()
            B.n_energies = t.n_energies
            B.lut_len = t.lut_len
            B.dvp_len = t.dvp_len
        # per-layer culling bounds (spot box, halo and MCS sigma bounds) on the device
        if self.layer_offsets[-1]:
            check(_lib.lib.pb_layer_bounds(ctypes.cast(self.beams, ctypes.c_void_p), self.n_beams,
                                           ptr(self.layers), ptr(self.spot_geo),
                                           _stream(self.device)), "pb_layer_bounds")
        self.spots_loaded = True

    def __del__(self):
        if not getattr(self, "_owns_textures", True):
            return
        for name in ("_tex", "_cells"):
            h = getattr(self, name, None)
            if h is not None and h.value:
                try:
                    torch.cuda.synchronize(self.device)
                    _lib.lib.pb_texture_destroy(h)
                except Exception:
                    pass
                h.value = 0

    # -- spot order helpers ---------------------------------------------------
    def to_sorted(self, mu_plan: torch.Tensor) -> torch.Tensor:
        """Plan-row-ordered weights -> sorted (layer) order."""
        return mu_plan.index_select(0, self.perm)

    def to_plan(self, v_sorted: torch.Tensor) -> torch.Tensor:
        out = torch.empty_like(v_sorted)
        out.index_copy_(0, self.perm, v_sorted)
        return out

    def mu_plan(self) -> torch.Tensor:
        return self.to_plan(self.mu_sorted)

    # -- WET ---------------------------------------------------------------------
    def _texture(self, rlsp: torch.Tensor, kind: str = "texture") -> int:
        """The plan's texture ("texture") or records-only ("cells") handle,
        created on first use and refilled from rlsp."""
        st = _stream(self.device)
        h = self._tex if kind == "texture" else self._cells
        if h.value:
            check(_lib.lib.pb_texture_update(h, ptr(rlsp), st), "pb_texture_update")
        elif kind == "texture":
            check(_lib.lib.pb_texture_create(ptr(rlsp), ctypes.byref(self.grid), ctypes.byref(h),
                                             st), "pb_texture_create")
        else:
            check(_lib.lib.pb_cells_create(ptr(rlsp), ctypes.byref(self.grid), ctypes.byref(h),
                                           st), "pb_cells_create")
        return h.value

    def compute_wet(self, rlsp: torch.Tensor, check_status: bool = True,
                    wet_mode: str = "texture") -> torch.Tensor:
        """Smoothed WET (cm) of every beam: n_beams x V on the device.

        wet_mode "texture" samples RLSP through the texture unit as the
        reference does; "exact" uses exact trilinear weights (the FP64
        oracle's arithmetic)."""
        if rlsp.dtype != torch.float32 or rlsp.device != self.device or rlsp.numel() != self.n_vox:
            raise ValueError("rlsp must be a float32 tensor of the grid's size on the plan's device")
        if wet_mode not in ("texture", "exact"):
            raise ValueError("wet_mode must be 'texture' or 'exact'")
        rlsp = rlsp.contiguous()
        tex = self._texture(rlsp, "texture" if wet_mode == "texture" else "cells")
        raw = torch.empty((self.n_beams, self.n_vox), dtype=torch.float32, device=self.device)
        wet = torch.empty_like(raw)
        self._status.zero_()
        check(_lib.lib.pb_wet(ptr(rlsp), tex, ctypes.byref(self.grid),
                              ctypes.cast(self.geoms, ctypes.c_void_p),
                              self.n_beams, ptr(raw), ptr(wet), ptr(self._status),
                              _stream(self.device)), "pb_wet")
        if check_status and int(self._status.item()) & _lib.PB_ERR_RAY_CAP:
            raise _lib.PbError(_lib.PB_ERR_RAY_CAP, "a WET ray reached its step cap")
        self.wet = wet
        self.raw_wet = raw
        self.wet_mode = wet_mode
        self._order = None
        self._beam_orders = None
        return wet

    def set_wet(self, wet: torch.Tensor) -> None:
        if wet.numel() != self.n_beams * self.n_vox or wet.dtype != torch.float32:
            raise ValueError("wet must be float32 with n_beams x V elements")
        self.wet = wet.to(self.device).reshape(self.n_beams, self.n_vox).contiguous()
        self._order = None
        self._beam_orders = None

    def _beam_ptr(self, b: int) -> ctypes.c_void_p:
        return ctypes.c_void_p(ctypes.addressof(self.beams) + b * ctypes.sizeof(PbBeam))

    def _make_order(self, beams: ctypes.c_void_p, n_beams: int,
                    wet: torch.Tensor) -> torch.Tensor:
        n = int(_lib.lib.pb_tile_order_count(ctypes.byref(self.grid)))
        size = int(_lib.lib.pb_tile_order_work_size(ctypes.byref(self.grid)))
        if self._order_work is None or self._order_work.numel() < size:
            self._order_work = torch.empty(size, dtype=torch.uint8, device=self.device)
        order = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
        check(_lib.lib.pb_tile_order(ctypes.byref(self.grid), beams, n_beams, ptr(wet),
                                     ptr(self.layers), ptr(self._order_work), ptr(order),
                                     _stream(self.device)), "pb_tile_order")
        return order

    def tile_order(self) -> torch.Tensor:
        """The default shape's tiles, most expensive first, for the current
        WET (pb_tile_order); computed once per WET, stream-ordered."""
        self._need_wet()
        if self._order is None:
            self._order = self._make_order(ctypes.cast(self.beams, ctypes.c_void_p),
                                           self.n_beams, self.wet)
        return self._order

    def beam_tile_order(self, b: int) -> torch.Tensor:
        """Beam b's tiles alone, most expensive first (pb_tile_order on that
        beam); computed once per WET, stream-ordered."""
        self._need_wet()
        if not 0 <= b < self.n_beams:
            raise IndexError(f"beam {b} of {self.n_beams}")
        if self._beam_orders is None:
            self._beam_orders = [None] * self.n_beams
        if self._beam_orders[b] is None:
            self._beam_orders[b] = self._make_order(self._beam_ptr(b), 1, self.wet[b])
        return self._beam_orders[b]

    def _need_wet(self):
        if not self.spots_loaded:
            raise RuntimeError("the plan's spots are not loaded (load_spots)")
        if self.wet is None:
            raise RuntimeError("WET has not been computed for this plan")

    # -- forward / adjoint -------------------------------------------------------
    def forward(self, mu_sorted: Optional[torch.Tensor] = None, scale: float = 1.0,
                beam_doses: bool = False, out: Optional[torch.Tensor] = None):
        """Dose (V) = scale * sum over beams; optionally n_beams x V per beam."""
        self._need_wet()
        mu = self.mu_sorted if mu_sorted is None else mu_sorted
        if mu.dtype != torch.float32 or mu.numel() != self.n_spots:
            raise ValueError("mu must be float32 with one entry per spot")
        mu = mu.contiguous()
        dose = out if out is not None else torch.empty(self.n_vox, dtype=torch.float32,
                                                       device=self.device)
        bd = torch.empty((self.n_beams, self.n_vox), dtype=torch.float32,
                         device=self.device) if beam_doses else None
        order = self.tile_order()
        check(_lib.lib.pb_dose_ordered(ctypes.byref(self.grid),
                                       ctypes.cast(self.beams, ctypes.c_void_p), self.n_beams,
                                       ptr(self.wet), ptr(self.layers), ptr(self.spot_geo),
                                       ptr(mu), float(scale), ptr(dose), ptr(bd), ptr(order),
                                       _stream(self.device)), "pb_dose_ordered")
        return (dose, bd) if beam_doses else dose

    def beam_tile_order_parts(self, b: int, n_parts: int):
        """Beam b's tile order split into up to n_parts groups of whole z
        slabs of tiles, lowest z first: a list of (order, v0, v1), each order
        the group's tiles most expensive first, padded with -1 to the full
        count (the kernel skips those entries), covering exactly voxels
        v0 <= v < v1 (z varies slowest).  One group when the grid has a
        single slab of tiles."""
        order = self.beam_tile_order(b)
        tile = (ctypes.c_int * 3)()
        check(_lib.lib.pb_tile_order_tile(tile), "pb_tile_order_tile")
        return split_order_by_slabs(order, (self.grid.nx, self.grid.ny, self.grid.nz),
                                    tuple(tile), n_parts)

    def forward_beam(self, b: int, mu_sorted: Optional[torch.Tensor] = None,
                     scale: float = 1.0, out: Optional[torch.Tensor] = None,
                     order: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Beam b's dose alone (V): the kernel run on that beam, in its own
        tile order; the same values as forward()'s per-beam dose of b.  With
        `order` (one of beam_tile_order_parts) only the tiles it lists are
        computed."""
        self._need_wet()
        mu = self.mu_sorted if mu_sorted is None else mu_sorted
        if mu.dtype != torch.float32 or mu.numel() != self.n_spots:
            raise ValueError("mu must be float32 with one entry per spot")
        mu = mu.contiguous()
        if order is None:
            order = self.beam_tile_order(b)
        elif (order.dtype != torch.int32 or order.device != self.device
              or order.numel() != self.beam_tile_order(b).numel()):
            raise ValueError("order must be an int32 device tensor of the full tile count")
        dose = out if out is not None else torch.empty(self.n_vox, dtype=torch.float32,
                                                       device=self.device)
        if dose.numel() != self.n_vox or not dose.is_contiguous():
            raise ValueError("out must be a contiguous tensor of V floats")
        check(_lib.lib.pb_dose_ordered(ctypes.byref(self.grid), self._beam_ptr(b), 1,
                                       ptr(self.wet[b]), ptr(self.layers), ptr(self.spot_geo),
                                       ptr(mu), float(scale), ptr(dose), None, ptr(order),
                                       _stream(self.device)), "pb_dose_ordered")
        return dose

    def forward_variant(self, variant: int, mu_sorted: Optional[torch.Tensor] = None,
                        scale: float = 1.0, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Forward dose with one of the kernel shapes of pb_dose_variant."""
        self._need_wet()
        mu = (self.mu_sorted if mu_sorted is None else mu_sorted).contiguous()
        dose = out if out is not None else torch.empty(self.n_vox, dtype=torch.float32,
                                                       device=self.device)
        check(_lib.lib.pb_dose_variant(ctypes.byref(self.grid),
                                       ctypes.cast(self.beams, ctypes.c_void_p), self.n_beams,
                                       ptr(self.wet), ptr(self.layers), ptr(self.spot_geo),
                                       ptr(mu), float(scale), ptr(dose), int(variant),
                                       _stream(self.device)), "pb_dose_variant")
        return dose

    def adjoint(self, dobj_ddose: torch.Tensor, scale: float = 1.0,
                out: Optional[torch.Tensor] = None,
                variant: Optional[int] = None) -> torch.Tensor:
        """grad[s] (sorted order) = scale * sum_v dobj_ddose[v] K(v, s).
        variant: the kernel family of that forward shape (default: the
        library's default shape)."""
        self._need_wet()
        if dobj_ddose.dtype != torch.float32 or dobj_ddose.numel() != self.n_vox:
            raise ValueError("dobj_ddose must be float32 with one entry per voxel")
        w = dobj_ddose.contiguous()
        grad = out if out is not None else torch.empty(max(self.n_spots, 1), dtype=torch.float32,
                                                       device=self.device)
        if variant is None:
            order = self.tile_order()
            check(_lib.lib.pb_dose_adjoint_ordered(
                ctypes.byref(self.grid), ctypes.cast(self.beams, ctypes.c_void_p), self.n_beams,
                ptr(self.wet), ptr(self.layers), ptr(self.spot_geo), ptr(w), float(scale),
                ptr(grad), ptr(order), _stream(self.device)), "pb_dose_adjoint_ordered")
        else:
            check(_lib.lib.pb_dose_adjoint_variant(
                ctypes.byref(self.grid), ctypes.cast(self.beams, ctypes.c_void_p), self.n_beams,
                ptr(self.wet), ptr(self.layers), ptr(self.spot_geo), ptr(w), float(scale),
                ptr(grad), int(variant), _stream(self.device)), "pb_dose_adjoint_variant")
        return grad[: self.n_spots]

    def adjoint_positions(self, dobj_ddose: torch.Tensor, scale: float = 1.0,
                          mu_sorted: Optional[torch.Tensor] = None):
        """(weight gradient, d/dx, d/dy) of sum_v dobj_ddose[v] D_v over the
        spots in sorted order, x and y the spot position at the isocentre
        plane (mm)."""
        self._need_wet()
        if dobj_ddose.dtype != torch.float32 or dobj_ddose.numel() != self.n_vox:
            raise ValueError("dobj_ddose must be float32 with one entry per voxel")
        mu = self.mu_sorted if mu_sorted is None else mu_sorted
        n = max(self.n_spots, 1)
        g, gx, gy = (torch.empty(n, dtype=torch.float32, device=self.device) for _ in range(3))
        check(_lib.lib.pb_dose_adjoint_positions(
            ctypes.byref(self.grid), ctypes.cast(self.beams, ctypes.c_void_p), self.n_beams,
            ptr(self.wet), ptr(self.layers), ptr(self.spot_geo), ptr(mu.contiguous()),
            ptr(dobj_ddose.contiguous()), float(scale), ptr(g), ptr(gx), ptr(gy),
            _stream(self.device)), "pb_dose_adjoint_positions")
        return g[: self.n_spots], gx[: self.n_spots], gy[: self.n_spots]

    def count_pairs(self) -> int:
        """Dense spot-voxel pair count E of the reference kernel."""
        self._need_wet()
        c = torch.zeros(1, dtype=torch.int64, device=self.device)
        check(_lib.lib.pb_count_pairs(ctypes.byref(self.grid), ctypes.cast(self.beams, ctypes.c_void_p),
                                      self.n_beams, ptr(self.wet), ptr(self.layers), ptr(c),
                                      _stream(self.device)), "pb_count_pairs")
        return int(c.item())


    def count_evaluated(self):
        """(SFU exp2 operations, spot-voxel evaluations) one forward issues,
        counted with the forward kernel's own culling decisions."""
        self._need_wet()
        c = torch.zeros(2, dtype=torch.int64, device=self.device)
        check(_lib.lib.pb_count_evaluated(ctypes.byref(self.grid),
                                          ctypes.cast(self.beams, ctypes.c_void_p), self.n_beams,
                                          ptr(self.wet), ptr(self.layers), ptr(self.spot_geo),
                                          ptr(c), _stream(self.device)), "pb_count_evaluated")
        v = c.cpu().tolist()
        return int(v[0]), int(v[1])

    def count_evaluated_adjoint(self, dobj_dose, scale: float = 1.0):
        """(SFU exp2 operations, spot-voxel evaluations) one adjoint on the
        field `dobj_dose` issues: the forward's decisions on the tiles the
        adjoint does not skip."""
        self._need_wet()
        if dobj_dose.dtype != torch.float32 or dobj_dose.numel() != self.n_vox:
            raise ValueError("dobj_dose must be float32 with one entry per voxel")
        w = dobj_dose.contiguous()
        c = torch.zeros(2, dtype=torch.int64, device=self.device)
        check(_lib.lib.pb_count_evaluated_adjoint(
            ctypes.byref(self.grid), ctypes.cast(self.beams, ctypes.c_void_p), self.n_beams,
            ptr(self.wet), ptr(self.layers), ptr(self.spot_geo), ptr(w), float(scale), ptr(c),
            _stream(self.device)), "pb_count_evaluated_adjoint")
        v = c.cpu().tolist()
        return int(v[0]), int(v[1])


def measure_ex2_rate(device) -> float:
    """Measured SFU exp2 throughput of a device (operations/s)."""
    device = require_cuda(device)
    r = ctypes.c_double(0.0)
    with torch.cuda.device(device):
        check(_lib.lib.pb_measure_ex2_rate(ctypes.byref(r), _stream(device)),
              "pb_measure_ex2_rate")
    return float(r.value)


_OBJ_WORK = {}


def objective(dose: torch.Tensor, presc: torch.Tensor, weight: torch.Tensor,
              resid: Optional[torch.Tensor] = None, out: Optional[torch.Tensor] = None):
    """FP64 sum_v w (D-P)^2 on the device (1-element float64 tensor, `out`
    if given) and, if ``resid`` is given, 2 w (D-P) written into it."""
    dev = dose.device
    n = dose.numel()
    for t in (presc, weight):
        if t.numel() != n or t.dtype != torch.float32 or t.device != dev:
            raise ValueError("dose, prescription and weights must match")
    work = _OBJ_WORK.get(dev)
    if work is None:
        work = torch.empty(int(_lib.lib.pb_objective_work_size()), dtype=torch.uint8, device=dev)
        _OBJ_WORK[dev] = work
    obj = out if out is not None else torch.empty(1, dtype=torch.float64, device=dev)
    check(_lib.lib.pb_objective(ptr(dose.contiguous()), ptr(presc.contiguous()),
                                ptr(weight.contiguous()), n, ptr(obj), ptr(resid), ptr(work),
                                _stream(dev)), "pb_objective")
    return obj


class HostGradientStep:
    """Objective and spot-weight gradient of a plan from pinned host
    buffers, the whole round trip of one optimiser step: the HU volume,
    prescription, voxel weights and spot weights go up, and the dose,
    gradient and objective come back.

    The copies off the critical path overlap the kernels:
    * the HU volume goes up first, alone, since the WET needs all of it;
    * the prescription and voxel weights follow on a copy stream while the
      WET and dose are computed (they are first read by the objective);
    * the dose comes back on the copy stream while the adjoint runs.
    The step ends, on the caller's current stream, once every copy has
    landed, so the next step may reuse every buffer.  Device buffers are
    allocated once, here.
    """

    def __init__(self, dp: DevicePlan, curve_hu: np.ndarray, curve_rlsp: np.ndarray,
                 wet_mode: str = "texture", scale: float = 1.0):
        self.dp = dp
        self.curve = (curve_hu, curve_rlsp)
        self.wet_mode = wet_mode
        self.scale = float(scale)
        dev = dp.device
        V = dp.n_vox
        f32 = dict(dtype=torch.float32, device=dev)
        self.hu = torch.empty(V, **f32)
        self.presc = torch.empty(V, **f32)
        self.weights = torch.empty(V, **f32)
        self.mu_plan = torch.empty(max(dp.n_spots, 1), **f32)
        self.rlsp = torch.empty(V, **f32)
        self.dose = torch.empty(V, **f32)
        self.resid = torch.empty(V, **f32)
        self.grad_sorted = torch.empty(max(dp.n_spots, 1), **f32)
        self.obj = torch.empty(1, dtype=torch.float64, device=dev)
        self.copy_stream = torch.cuda.Stream(dev)
        self._ev = {k: torch.cuda.Event() for k in ("hu", "inputs", "dose", "out")}

    def __call__(self, hu_h: torch.Tensor, presc_h: torch.Tensor, weights_h: torch.Tensor,
                 mu_plan_h: torch.Tensor, dose_out: torch.Tensor, grad_out: torch.Tensor,
                 obj_out: torch.Tensor) -> None:
        """Enqueue one step on the current stream.  Host tensors are pinned
        float32 (obj_out float64), V / n_spots elements, spot weights and the
        gradient in plan row order.  Nothing is synchronised: read the
        outputs after synchronising the current stream."""
        dp = self.dp
        n = dp.n_spots
        for name, t, m in (("hu", hu_h, dp.n_vox), ("prescription", presc_h, dp.n_vox),
                           ("voxel weights", weights_h, dp.n_vox), ("dose_out", dose_out, dp.n_vox),
                           ("spot weights", mu_plan_h, n), ("grad_out", grad_out, n)):
            if t.numel() != m or t.dtype != torch.float32 or t.device.type != "cpu":
                raise ValueError(f"{name} must be a host float32 tensor of {m} elements")
        if obj_out.numel() != 1 or obj_out.dtype != torch.float64 or obj_out.device.type != "cpu":
            raise ValueError("obj_out must be a host float64 tensor of one element")
        main = torch.cuda.current_stream(dp.device)
        cs, ev = self.copy_stream, self._ev
        # the copy stream may overwrite the inputs once the previous step's
        # kernels (queued on `main`) are done with them
        cs.wait_stream(main)
        self.hu.copy_(hu_h, non_blocking=True)
        ev["hu"].record(main)
        self.mu_plan[:n].copy_(mu_plan_h, non_blocking=True)
        with torch.cuda.stream(cs):
            cs.wait_event(ev["hu"])
            self.presc.copy_(presc_h, non_blocking=True)
            self.weights.copy_(weights_h, non_blocking=True)
            ev["inputs"].record(cs)
        rlsp_from_hu(self.hu, *self.curve, out=self.rlsp)
        dp.compute_wet(self.rlsp, check_status=False, wet_mode=self.wet_mode)
        dp.forward(dp.to_sorted(self.mu_plan[:n]), scale=self.scale, out=self.dose)
        ev["dose"].record(main)
        main.wait_event(ev["inputs"])
        objective(self.dose, self.presc, self.weights, self.resid, out=self.obj)
        with torch.cuda.stream(cs):
            cs.wait_event(ev["dose"])
            dose_out.copy_(self.dose, non_blocking=True)
            ev["out"].record(cs)
        dp.adjoint(self.resid, scale=self.scale, out=self.grad_sorted[:n])
        grad_out.copy_(dp.to_plan(self.grad_sorted[:n]), non_blocking=True)
        obj_out.copy_(self.obj, non_blocking=True)
        main.wait_event(ev["out"])
