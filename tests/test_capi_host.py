"""The C-ABI library on the host: it loads, exports every entry point the
header declares, its host-side plan preparation matches the oracle bit for
bit, and bad arguments come back as status codes (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pb_b200.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from dosecuda_b200 import _lib
    names = _declared()
    assert len(names) >= 16
    raw = ctypes.CDLL(_lib.LIB_PATH)
    for n in names:
        assert hasattr(raw, n), n
    assert set(names) <= set(_lib.EXPORTED)
    assert b"sm_100a" in _lib.lib.pb_version()


@pytest.mark.parametrize("gantry,couch", [(0, 0), (90, 0), (180, 0), (270, 0), (120, 0),
                                          (240, 0), (45, 90), (-90, 15), (359.5, 270),
                                          (33.3, -20)])
def test_beam_setup_matches_oracle_bitwise(gantry, couch, oracle):
    from dosecuda_b200 import _lib
    iso = np.array([12.5, -3.25, 40.0], np.float32)
    origin = np.array([-150.0, -151.5, -120.25], np.float32)
    g = _lib.beam_setup(gantry, couch, 1340.0, 1930.0, iso, origin)
    o = oracle.beam_setup(gantry, couch, 1340.0, 1930.0, iso, origin)
    assert bytes(g) == bytes(o)


def test_beam_setup_semantics():
    """gantry' = fmod(gantry + 180, 360); source at (VSADX+VSADY)/2 from iso."""
    from dosecuda_b200 import _lib
    g = _lib.beam_setup(0.0, 0.0, 1340.0, 1930.0, [0, 0, 0], [0, 0, 0])
    assert abs(g.src[1] + 1635.0) < 1e-3 and abs(g.src[0]) < 1e-3
    g = _lib.beam_setup(90.0, 0.0, 1340.0, 1930.0, [1, 2, 3], [0.5, 0.5, 0.5])
    assert list(g.iso) == [0.5, 1.5, 2.5]
    assert abs(np.hypot(g.src[0], g.src[1]) - 1635.0) < 1e-2


def _random_spots(rng, n, n_e):
    sl = np.zeros((n, 4), np.float32)
    sl[:, 0] = rng.uniform(-80, 80, n)
    sl[:, 1] = rng.uniform(-80, 80, n)
    sl[:, 2] = rng.uniform(0.1, 2.0, n)
    sl[:, 3] = rng.integers(0, n_e, n)
    return sl


def test_build_layers_matches_oracle(oracle):
    from dosecuda_b200 import _lib
    from dosecuda_b200.plan_impt import IMPTPlan
    dvp = IMPTPlan().beam_models[0].divergence_params
    rng = np.random.default_rng(0)
    for n in (0, 1, 7, 500):
        sl = _random_spots(rng, n, dvp.shape[0])
        s1, l1, perm = _lib.build_layers(sl, dvp)
        s2, l2 = oracle.build_layers(sl, dvp)
        assert s1.tobytes() == s2.tobytes()
        # the reference's five layer fields; the culling bounds are left unset
        assert len(l1) == len(l2)
        for f in ("spot_start", "n_spots", "energy_id", "r80", "energy"):
            assert np.array_equal(l1[f], l2[f])
        assert not l1["bound_ok"].any()
        # perm maps each sorted spot to its input row
        if n:
            assert np.array_equal(sl[perm][:, 0], s1["x"])


def test_build_layers_reference_quirks():
    """importLayers (IMPTClasses.cu:37-67): ids are truncated to int; ids at
    or above n_energies are dropped; one negative id blocks every layer."""
    from dosecuda_b200 import _lib
    dvp = np.zeros((5, 5), np.float32)
    dvp[:, 1] = [10, 20, 30, 40, 50]
    sl = np.array([[0, 0, 1, 3.9], [1, 0, 1, 1.0], [2, 0, 1, 7.0], [3, 0, 1, 1.2]], np.float32)
    spots, layers, perm = _lib.build_layers(sl, dvp)
    assert [(L["energy_id"], L["n_spots"], L["spot_start"]) for L in layers] == [(1, 2, 0),
                                                                                 (3, 1, 2)]
    assert list(perm) == [1, 3, 0, 2]
    assert layers[1]["r80"] == 40
    sl[0, 3] = -2.0
    _, layers, _ = _lib.build_layers(sl, dvp)
    assert len(layers) == 0


def test_spot_geometry_values():
    from dosecuda_b200 import _lib
    spots = np.zeros(3, _lib.SPOT_DTYPE)
    spots["x"] = [10.0, -20.0, 0.0]
    spots["y"] = [5.0, 7.5, 0.0]
    geo = _lib.spot_geometry(spots, 1340.0, 1930.0)
    x, y = spots["x"].astype(np.float64), spots["y"].astype(np.float64)
    tx, ty = x / 1340.0, y / 1930.0
    assert np.allclose(geo[:, 3], tx, rtol=1e-7) and np.allclose(geo[:, 4], ty, rtol=1e-7)
    assert np.allclose(geo[:, 5], x * y * (1 / 1340.0 - 1 / 1930.0), rtol=1e-6)
    assert np.allclose(geo[:, 2], 1.0 / (1.0 + tx * tx + ty * ty), rtol=1e-7)


def test_invalid_arguments_return_status_without_a_gpu():
    from dosecuda_b200 import _lib
    L = _lib.lib
    g = _lib.PbGrid(0, 4, 4, 2.0)
    assert L.pb_dose(ctypes.byref(g), None, 1, None, None, None, None, 1.0, None, None,
                     None) == _lib.PB_ERR_INVALID
    assert "dimensions" in _lib.last_error()
    g = _lib.PbGrid(4, 4, 4, 2.0)
    assert L.pb_dose(ctypes.byref(g), None, 0, None, None, None, None, 1.0, None, None,
                     None) == _lib.PB_ERR_INVALID
    assert L.pb_wet(None, 0, ctypes.byref(g), None, 1, None, None, None, None) == _lib.PB_ERR_INVALID
    g = _lib.PbGrid(4, 4, 4, -1.0)
    assert L.pb_wet(None, 0, ctypes.byref(g), None, 1, None, None, None, None) == _lib.PB_ERR_INVALID
    xh = np.array([0.0, 0.0], np.float64)
    yh = np.array([1.0, 2.0], np.float64)
    assert L.pb_rlsp_from_hu(ctypes.c_void_p(1), 4, _lib.ptr(xh), _lib.ptr(yh), 2,
                             ctypes.c_void_p(1), None) == _lib.PB_ERR_INVALID
    assert "increasing" in _lib.last_error()
    assert L.pb_objective(None, None, None, 4, None, None, None, None) == _lib.PB_ERR_INVALID
    assert L.pb_objective_work_size() >= 8
    dims = np.array([0, 4, 4], np.int64)
    buf = np.zeros(16, np.float32)
    assert L.pb_proton_raytrace_host(0, 1340.0, 1930.0, _lib.ptr(buf), _lib.ptr(dims),
                                     ctypes.c_float(2.0), _lib.ptr(buf), _lib.ptr(buf), 0.0, 0.0,
                                     _lib.ptr(buf)) == _lib.PB_ERR_INVALID
    # the tile order: sizes from the grid alone; bad grids, beams or buffers
    # are rejected before any device work
    g = _lib.PbGrid(256, 256, 160, 2.0)
    n = L.pb_tile_order_count(ctypes.byref(g))
    assert n == 32 * 16 * 20                          # 8 x 16 x 8 voxel tiles
    # page-locking a host range: NULL or empty ranges are refused without a
    # CUDA call
    assert L.pb_host_register(None, 4096) == _lib.PB_ERR_INVALID
    buf = (ctypes.c_char * 4096)()
    assert L.pb_host_register(buf, 0) == _lib.PB_ERR_INVALID
    assert L.pb_host_unregister(None) == _lib.PB_ERR_INVALID
    tile = (ctypes.c_int * 3)()
    assert L.pb_tile_order_tile(tile) == _lib.PB_OK and list(tile) == [8, 16, 8]
    assert L.pb_tile_order_tile(None) == _lib.PB_ERR_INVALID
    assert L.pb_tile_order_work_size(ctypes.byref(g)) >= 4 * n + 4096
    bad = _lib.PbGrid(0, 4, 4, 2.0)
    assert L.pb_tile_order_count(ctypes.byref(bad)) == -1
    assert L.pb_tile_order_work_size(ctypes.byref(bad)) == 0
    assert L.pb_tile_order(ctypes.byref(bad), None, 1, None, None, None, None,
                           None) == _lib.PB_ERR_INVALID
    assert L.pb_tile_order(ctypes.byref(g), None, 0, None, None, None, None,
                           None) == _lib.PB_ERR_INVALID
    assert L.pb_dose_ordered(ctypes.byref(g), None, 1, None, None, None, None, 1.0, None, None,
                             None, None) == _lib.PB_ERR_INVALID
    assert L.pb_dose_adjoint_ordered(ctypes.byref(g), None, 1, None, None, None, None, 1.0,
                                     None, None, None) == _lib.PB_ERR_INVALID


def _smoothing_cases(n):
    """Beams over small grids; every third case puts the grid and the
    isocentre far from the coordinate origin (hundreds of mm), where the
    FP32 positions round more coarsely."""
    rng = np.random.default_rng(17)
    spacings = [1.0, 1.5, 2.0, 2.5, 3.0, 0.9765625, 1.171875, 2.34375, 1.2]
    for c in range(n):
        gantry = [0.0, 90.0, 180.0, 270.0][c % 4] if c % 2 == 0 else float(rng.uniform(0, 360))
        couch = [0.0, 90.0, 270.0, float(rng.uniform(-90, 90))][(c // 2) % 4]
        s = spacings[c % len(spacings)]
        shape = tuple(int(x) for x in rng.integers(8, 22, 3))
        if c % 3 == 2:
            iso = rng.uniform(-400, 400, 3).astype(np.float32)
            origin = rng.uniform(-700, 700, 3).astype(np.float32)
        else:
            iso = rng.uniform(-100, 100, 3).astype(np.float32)
            origin = (-(np.array(shape[::-1]) * s) / 2 + rng.uniform(-20, 20, 3)).astype(np.float32)
        yield gantry, couch, s, shape, iso, origin


def test_smoothing_table_holds_the_reference_samples(oracle):
    """The WET pass's smoothing table (pb_smooth_table) against the voxels
    the reference's FP32 arithmetic picks (oracle), for every sample of
    every voxel, over 180 beams: axis-aligned and oblique gantries, couch
    rotations, 9 spacings (powers of two and not), random isocentres, a
    third of them hundreds of mm from the origin.  An
    unflagged sample is exactly the table's voxel; a flagged one (a
    half-voxel tie) is that voxel or the next; the linear offsets agree with
    the per-axis ones; inside the margins every candidate is in the grid."""
    from dosecuda_b200 import _lib
    n_flag = 0
    for gantry, couch, s, shape, iso, origin in _smoothing_cases(180):
        geom = _lib.beam_setup(gantry, couch, 1340.0, 1930.0, iso, origin)
        ob = oracle.beam_setup(gantry, couch, 1340.0, 1930.0, iso, origin)
        off, hh, tmask, margin = _lib.smooth_table(shape, s, [geom], 0)
        ro = np.floor(hh).astype(np.int64)
        assert np.array_equal(hh, ro + 0.5)
        nz, ny, nx = shape
        assert np.array_equal(off, ro[..., 0] + nx * ro[..., 1] + nx * ny * ro[..., 2])
        bit = 3 * np.arange(9)[:, None] + np.arange(3)[None, :]
        flag = ((tmask[:, None, None] >> bit[None]) & 1).astype(bool)      # [6, 9, 3]
        n_flag += int(flag.sum())
        got = oracle.smooth_choices(shape, s, ob).astype(np.int64)        # [z, y, x, 6, 9, 3]
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        own = np.stack([i, j, k], -1)[:, :, :, None, None, :]
        step = got - (own + ro)
        assert np.all(step[..., ~flag] == 0), (gantry, couch, s)
        assert np.all((step[..., flag] == 0) | (step[..., flag] == 1)), (gantry, couch, s)
        n = np.array([nx, ny, nz])
        lo_ok = own[..., 0, 0, :] - margin >= 0
        hi_ok = own[..., 0, 0, :] + margin <= n - 1
        inner = np.all(lo_ok & hi_ok, -1)
        if inner.any():
            cand_lo = (own + ro)[inner]
            cand_hi = cand_lo + flag
            assert cand_lo.min() >= 0 and np.all(cand_hi <= n - 1)
    assert n_flag > 0   # the axis-aligned beams do have ties


def test_smoothing_table_rejects_bad_arguments():
    from dosecuda_b200 import _lib
    geom = _lib.beam_setup(0.0, 0.0, 1340.0, 1930.0, [0, 0, 0], [0, 0, 0])
    with pytest.raises(_lib.PbError):
        _lib.smooth_table((10, 10, 10), 2.0, [geom], 1)
    with pytest.raises(_lib.PbError):
        _lib.smooth_table((10, 0, 10), 2.0, [geom], 0)


@pytest.mark.parametrize("dims,n_parts", [((256, 256, 160), 4), ((56, 48, 40), 2),
                                          ((56, 48, 40), 9), ((20, 17, 7), 4),
                                          ((33, 40, 41), 3)])
def test_tile_order_split_by_z_slabs(dims, n_parts):
    """The split computeIMPTPlan uses for a plan's last beam: groups of whole
    z slabs of tiles, in the given order within each group, -1 padded, each
    covering exactly its voxel range (host logic, CPU tensors)."""
    import torch
    from dosecuda_b200.engine import split_order_by_slabs
    tile = (8, 16, 8)
    nx, ny, nz = dims
    tx, ty, tz = (-(-nx // tile[0]), -(-ny // tile[1]), -(-nz // tile[2]))
    n = tx * ty * tz
    order = torch.randperm(n, generator=torch.Generator().manual_seed(n)).to(torch.int32)
    parts = split_order_by_slabs(order, dims, tile, n_parts)
    assert len(parts) == min(n_parts, tz)
    assert parts[0][1] == 0 and parts[-1][2] == nx * ny * nz
    seen = []
    for (o, v0, v1), nxt in zip(parts, parts[1:] + [None]):
        assert o.numel() == n and o.dtype == torch.int32
        listed = o[o >= 0]
        assert bool((o[listed.numel():] == -1).all())
        # the group's tiles in the order's own sequence
        pos = torch.empty(n, dtype=torch.long)
        pos[order.long()] = torch.arange(n)
        assert bool((pos[listed.long()].diff() > 0).all()) if listed.numel() > 1 else True
        # exactly the tiles whose z slab lies in [v0, v1)
        slabs = listed // (tx * ty)
        assert v0 == nx * ny * min(int(slabs.min()) * tile[2], nz)
        assert v1 == nx * ny * min((int(slabs.max()) + 1) * tile[2], nz)
        assert listed.numel() == (int(slabs.max()) - int(slabs.min()) + 1) * tx * ty
        if nxt is not None:
            assert nxt[1] == v1
        seen.append(listed)
    allt = torch.cat(seen).sort().values
    assert torch.equal(allt, torch.arange(n, dtype=torch.int32))
