"""pb_wet_noalloc: the WET pass for callers that cannot allocate device memory.

Some callers of this library cannot call cudaMalloc: code running inside a
framework that owns the device pool (an XLA/JAX custom call, whose allocator
has already reserved most of the GPU and which hands the call only its input
and output buffers) or a plug-in given only its buffers.  pb_wet_noalloc
keeps its work space in a fixed array inside the library instead of taking
one from the caller.  This test calls it through the C-ABI twice in a row
and checks each result against pb_wet with a caller-provided work buffer.
Both run the same kernels on the same inputs, so the results must be equal
bit for bit (tighter than the 1e-4 cm of the other WET tests).  Between the
two calls, a call on a larger grid with other RLSP values leaves different
contents in the shared work array: a read of anything the second call did
not write first would change its bits.  A request larger than the fixed
work space, and a grid that pb_wet rejects, are refused with a clear error.

The file name sorts last so that a run stopping at the first failure has run
every other test first; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _inputs():
    import torch

    from dosecuda_b200 import _lib, engine, phantoms
    from dosecuda_b200.plan_impt import _hu_curve
    case = phantoms.small_heterogeneous()
    g, plan = case.grid, case.plan
    dev = torch.device("cuda", 0)
    hu = torch.from_numpy(np.ascontiguousarray(g.HU).reshape(-1)).to(dev)
    rlsp = engine.rlsp_from_hu(hu, *_hu_curve(plan.machine_name))
    grid = engine.grid_of(g.HU.shape, float(g.spacing[0]))
    n = len(plan.beam_list)
    geoms = (_lib.PbBeamGeom * n)()
    for b, beam in enumerate(plan.beam_list):
        m = plan.beam_models[0]
        geoms[b] = _lib.beam_setup(beam.gantry_angle, beam.couch_angle, m.VSADX, m.VSADY,
                                   beam.iso, np.asarray(g.origin, np.float32))
    return torch, _lib, dev, rlsp, grid, geoms, n, int(np.prod(g.HU.shape))


@pytest.mark.parametrize("mode", ["exact", "texture"])
def test_wet_noalloc_matches_pb_wet_on_two_calls(mode):
    torch, L, dev, rlsp, grid, geoms, n, V = _inputs()
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    tex = ctypes.c_uint64(0)
    if mode == "texture":
        L.check(L.lib.pb_texture_create(L.ptr(rlsp), ctypes.byref(grid), ctypes.byref(tex),
                                        stream))
    try:
        raw = torch.empty(n * V, dtype=torch.float32, device=dev)
        want = torch.empty(n * V, dtype=torch.float32, device=dev)
        L.check(L.lib.pb_wet(L.ptr(rlsp), tex.value, ctypes.byref(grid),
                             ctypes.cast(geoms, ctypes.c_void_p), n, L.ptr(raw), L.ptr(want),
                             None, stream))
        for call in range(2):
            got = torch.full((n * V,), -1.0, dtype=torch.float32, device=dev)
            status = torch.zeros(1, dtype=torch.int32, device=dev)
            L.check(L.lib.pb_wet_noalloc(L.ptr(rlsp), tex.value, ctypes.byref(grid),
                                         ctypes.cast(geoms, ctypes.c_void_p), n, L.ptr(got),
                                         L.ptr(status), stream))
            torch.cuda.synchronize(dev)
            assert int(status.item()) == 0
            assert torch.equal(got, want)
            if call == 0:
                _fill_work_array_with_another_grid(torch, L, dev, grid, geoms, n, stream)
    finally:
        torch.cuda.synchronize(dev)
        if tex.value:
            L.lib.pb_texture_destroy(tex)


def _fill_work_array_with_another_grid(torch, L, dev, grid, geoms, n, stream):
    """A pb_wet_noalloc call on a larger grid (8 more voxels per axis) with
    dense random RLSP: the shared work array then holds other raw WET
    values over (and past) the region the next call uses."""
    big = L.PbGrid(grid.nx + 8, grid.ny + 8, grid.nz + 8, grid.spacing)
    Vb = big.nx * big.ny * big.nz
    assert n * Vb <= L.PB_NOALLOC_MAX_WET_FLOATS
    rng = torch.Generator(device=dev).manual_seed(9)
    rlsp_big = torch.rand(Vb, generator=rng, device=dev) * 3.0 + 0.5
    out = torch.empty(n * Vb, dtype=torch.float32, device=dev)
    L.check(L.lib.pb_wet_noalloc(L.ptr(rlsp_big), 0, ctypes.byref(big),
                                 ctypes.cast(geoms, ctypes.c_void_p), n, L.ptr(out), None,
                                 stream))
    torch.cuda.synchronize(dev)


def test_wet_noalloc_rejects_requests_beyond_its_work_space():
    torch, L, dev, rlsp, grid, geoms, n, V = _inputs()
    big = L.PbGrid(256, 256, 129, 2.0)   # 8.45 M voxels > 8 Mi floats for one beam
    out = torch.empty(1, dtype=torch.float32, device=dev)
    status = L.lib.pb_wet_noalloc(L.ptr(rlsp), 0, ctypes.byref(big),
                                  ctypes.cast(geoms, ctypes.c_void_p), 1, L.ptr(out), None,
                                  None)
    assert status == L.PB_ERR_INVALID
    assert "exceeds its fixed work space" in L.last_error()
    # a grid that pb_wet rejects is rejected here too (the same checks)
    bad = L.PbGrid(grid.nx, grid.ny, grid.nz, float("inf"))
    for fn, extra in ((L.lib.pb_wet_noalloc, ()), (L.lib.pb_wet, (L.ptr(out),))):
        args = [L.ptr(rlsp), 0, ctypes.byref(bad), ctypes.cast(geoms, ctypes.c_void_p), n]
        args += list(extra) + [L.ptr(out), None, None]
        assert fn(*args) == L.PB_ERR_INVALID
        assert "spacing" in L.last_error()
