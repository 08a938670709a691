"""pb_wet_noalloc: the WET pass for callers that cannot allocate device memory.

Some callers of this library cannot call cudaMalloc: code running inside a
framework that owns the device pool (an XLA/JAX custom call, whose allocator
has already reserved most of the GPU and which hands the call only its input
and output buffers) or a plug-in given only its buffers.  pb_wet_noalloc
keeps its work space in a fixed array inside the library instead of taking
one from the caller.  This test calls it through the C-ABI twice in a row
and checks each result against pb_wet with a caller-provided work buffer
(same inputs; the same tolerance as the other WET tests, 1e-4 cm), and that
a request larger than the fixed work space is refused with a clear error.

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
        for _ in range(2):
            got = torch.full((n * V,), -1.0, dtype=torch.float32, device=dev)
            status = torch.zeros(1, dtype=torch.int32, device=dev)
            L.check(L.lib.pb_wet_noalloc(L.ptr(rlsp), tex.value, ctypes.byref(grid),
                                         ctypes.cast(geoms, ctypes.c_void_p), n, L.ptr(got),
                                         L.ptr(status), stream))
            torch.cuda.synchronize(dev)
            assert int(status.item()) == 0
            assert float((got - want).abs().max()) <= 1e-4
    finally:
        torch.cuda.synchronize(dev)
        if tex.value:
            L.lib.pb_texture_destroy(tex)


def test_wet_noalloc_rejects_requests_beyond_its_work_space():
    torch, L, dev, rlsp, grid, geoms, n, V = _inputs()
    big = L.PbGrid(256, 256, 129, 2.0)   # 8.45 M voxels > 8 Mi floats for one beam
    out = torch.empty(1, dtype=torch.float32, device=dev)
    status = L.lib.pb_wet_noalloc(L.ptr(rlsp), 0, ctypes.byref(big),
                                  ctypes.cast(geoms, ctypes.c_void_p), 1, L.ptr(out), None,
                                  None)
    assert status == L.PB_ERR_INVALID
    assert "exceeds its fixed work space" in L.last_error()
