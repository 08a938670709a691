"""Parity of the CUDA path with the FP64 oracle and with the reference's own
CUDA module (oracle/_ref), through the package's C-ABI.

Tolerances (fractions of the reference dose maximum Dmax unless stated):
  * exact-trilinear WET vs FP64 oracle:          |dWET| <= 1e-4 cm
  * dose vs FP64 oracle (same decisions):         <= 1e-3 Dmax  (0.1 %)
  * pencil-beam pass alone (same WET):            <= 2e-4 Dmax
  * texture-mode WET / dose vs reference module:  <= 1e-3 Dmax
  * spot-weight gradient vs central differences:  <= 1e-3 of max |g|
"""
import numpy as np
import pytest
import torch

from conftest import cuda_available, max_rel

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DEV = torch.device("cuda", 0)


@pytest.fixture(scope="module")
def pkg():
    import dosecuda_b200
    from dosecuda_b200 import engine, phantoms, plan_impt
    return dosecuda_b200, engine, phantoms, plan_impt


@pytest.fixture(scope="module")
def curve(pkg):
    return pkg[3]._hu_curve("HitachiProbeatJHU")


@pytest.fixture(scope="module")
def small(pkg):
    return pkg[2].small_heterogeneous()


@pytest.fixture(scope="module")
def cube(pkg):
    return pkg[2].water_cube()


def _vol(data, grid):
    from dosecuda_b200.plan import VolumeObject
    v = VolumeObject()
    v.voxel_data = np.ascontiguousarray(data, np.float32)
    v.origin = np.array(grid.origin, np.float32)
    v.spacing = np.array(grid.spacing, np.float32)
    return v


def _model(plan, beam):
    labels = list(plan.dicom_rangeshifter_label.astype(str))
    return plan.beam_models[labels.index(beam.dicom_rangeshifter_label)]


def _oracle_beam(O, grid, beam, model):
    m = O.Model(model)
    ob = O.beam_setup(beam.gantry_angle, beam.couch_angle, m.vsadx, m.vsady, beam.iso,
                      grid.origin)
    spots, layers = O.build_layers(np.asarray(beam.spot_list, np.float32).reshape(-1, 4), m.dvp)
    return m, ob, spots, layers


# ----------------------------------------------------------------- HU->RLSP

def test_rlsp_bitwise_numpy_interp(pkg, curve):
    engine = pkg[1]
    rng = np.random.default_rng(0)
    hu = np.concatenate([rng.uniform(-1500, 4000, 200000).astype(np.float32),
                         curve[0].astype(np.float32),
                         np.array([-1e6, 1e6, 0.0, -1000.0, 3096.0, 1369.0], np.float32)])
    got = engine.rlsp_from_hu(torch.from_numpy(hu).to(DEV), *curve).cpu().numpy()
    want = np.array(np.interp(hu, *curve), dtype=np.single)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


# ------------------------------------------------------- exact mode vs oracle

def test_wet_exact_matches_oracle(pkg, small, curve, oracle):
    g = small.grid
    dp = g.prepareIMPTPlan(small.plan, 0, wet_mode="exact")
    wet = dp.wet.cpu().numpy().reshape(dp.n_beams, *g.HU.shape)
    rlsp = oracle.rlsp_from_hu(g.HU, *curve)
    for b, beam in enumerate(small.plan.beam_list):
        _, ob, _, _ = _oracle_beam(oracle, g, beam, _model(small.plan, beam))
        raw = oracle.raytrace(rlsp, g.spacing[0], ob).astype(np.float32)
        sm = oracle.smooth(raw, g.spacing[0], ob)
        assert np.abs(wet[b] - sm).max() <= 1e-4


@pytest.mark.parametrize("which", ["small", "full"])
def test_exact_wet_runs_match_sample_by_sample(pkg, small, curve, which):
    """Exact-trilinear WET with the cell records (pb_cells_create: runs
    through flat cells) against the same pass sampling every step (handle
    0): equal up to the FP64 summation order; a sample taken from a wrong
    cell would show as >= 1e-2 cm."""
    import ctypes
    from dosecuda_b200 import _lib, engine
    case = small if which == "small" else pkg[2].config_gradient()
    g = case.grid
    dp = g.prepareIMPTPlan(case.plan, 0, wet_mode="exact")
    runs = dp.wet.clone()
    hu = torch.from_numpy(np.ascontiguousarray(g.HU).reshape(-1)).to(DEV)
    rlsp = engine.rlsp_from_hu(hu, *curve)
    raw = torch.empty_like(runs)
    each = torch.empty_like(runs)
    _lib.check(_lib.lib.pb_wet(_lib.ptr(rlsp), 0, ctypes.byref(dp.grid),
                               ctypes.cast(dp.geoms, ctypes.c_void_p), dp.n_beams, _lib.ptr(raw),
                               _lib.ptr(each), None,
                               ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)))
    torch.cuda.synchronize(DEV)
    assert float((runs - each).abs().max()) <= 1e-4


def test_dose_exact_matches_oracle(pkg, small, cube, curve, oracle):
    for case in (small, cube):
        g, plan = case.grid, case.plan
        dp = g.prepareIMPTPlan(plan, 0, wet_mode="exact")
        dose, bd = dp.forward(beam_doses=True)
        bd = bd.cpu().numpy().reshape(dp.n_beams, *g.HU.shape)
        beams = [(b.gantry_angle, b.couch_angle, b.iso, b.spot_list, _model(plan, b))
                 for b in plan.beam_list]
        ref = oracle.plan_forward(g.HU, g.origin, g.spacing[0], beams, curve)
        assert max_rel(dose.cpu().numpy().reshape(g.HU.shape), ref["dose"]) <= 1e-3
        for b in range(dp.n_beams):
            assert max_rel(bd[b], ref["beam_dose"][b]) <= 1e-3


def test_pencil_beam_pass_matches_oracle_same_wet(pkg, small, oracle):
    engine = pkg[1]
    g, plan = small.grid, small.plan
    dp = g.prepareIMPTPlan(plan, 0, wet_mode="exact")
    wet = dp.wet.cpu().numpy().reshape(dp.n_beams, *g.HU.shape)
    bd = dp.forward(beam_doses=True)[1].cpu().numpy().reshape(dp.n_beams, *g.HU.shape)
    for b, beam in enumerate(plan.beam_list):
        m, ob, spots, layers = _oracle_beam(oracle, g, beam, _model(plan, beam))
        want = oracle.dose(wet[b], g.spacing[0], ob, m, spots, layers)
        assert max_rel(bd[b], want) <= 2e-4
    del engine


# ------------------------------------------- texture mode vs the reference

def _reference_plan(ref, case, curve):
    g, plan = case.grid, case.plan
    rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
    wets, doses = [], []
    for beam in plan.beam_list:
        model = _model(plan, beam)
        w = ref.proton_raytrace_cuda(model, _vol(rlsp, g), beam, 0)
        beam.spot_list = np.asarray(beam.spot_list, np.float32).reshape(-1, 4)
        d = ref.proton_spot_cuda(model, _vol(rlsp, g), _vol(w, g), beam, 0)
        wets.append(w)
        doses.append(d)
    return wets, doses


def test_texture_mode_matches_reference(pkg, small, cube, curve, reference_module):
    for case in (small, cube):
        g = case.grid
        dp = g.prepareIMPTPlan(case.plan, 0, wet_mode="texture")
        wet = dp.wet.cpu().numpy().reshape(dp.n_beams, *g.HU.shape)
        bd = dp.forward(beam_doses=True)[1].cpu().numpy().reshape(dp.n_beams, *g.HU.shape)
        rw, rd = _reference_plan(reference_module, case, curve)
        for b in range(dp.n_beams):
            # the reference sums its samples in FP32, this path in FP64: on
            # these short rays they differ by < 7e-5 cm everywhere; a sample
            # taken from a wrong cell would show as >= 1e-2 cm
            assert np.abs(wet[b] - rw[b]).max() <= 1e-4
            assert max_rel(bd[b], rd[b]) <= 1e-3


@pytest.mark.parametrize("gantry,couch", [(0.0, 0.0), (90.0, 0.0), (33.0, 20.0)])
def test_smoothing_ties_match_reference(pkg, curve, reference_module, gantry, couch):
    """At 2 mm with the beam along an image axis, every other radius of two
    smoothing directions lands exactly on a half-voxel, where the chosen
    voxel follows the reference's FP32 rounding; an oblique beam has no such
    ties.  Texture-mode WET against the reference module at every voxel."""
    case = pkg[2].heterogeneous(11, (gantry,), 60, shape=(48, 80, 72), spacing=2.0,
                                n_slabs=1, n_spheres=2, semi_range=(10.0, 14.0),
                                centre_jitter=4.0, body_inset=12.0)
    beam = case.plan.beam_list[0]
    beam.couch_angle = couch
    g = case.grid
    dp = g.prepareIMPTPlan(case.plan, 0, wet_mode="texture")
    wet = dp.wet.cpu().numpy().reshape(g.HU.shape)
    rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
    want = reference_module.proton_raytrace_cuda(_model(case.plan, beam), _vol(rlsp, g), beam, 0)
    assert np.abs(wet - want).max() <= 1e-4


@pytest.mark.parametrize("gantry,couch,spacing", [(0.0, 0.0, 2.0), (90.0, 0.0, 2.0),
                                                 (270.0, 90.0, 2.5), (33.3, 15.0, 3.0),
                                                 (180.0, 0.0, 1.5), (225.0, 300.0, 2.0),
                                                 (90.0, 0.0, 3.0), (0.0, 0.0, 1.0)])
def test_smoothing_bitwise_reference_arithmetic(pkg, oracle, gantry, couch, spacing):
    """The smoothing alone, bit for bit: the kernel's raw WET of a noisy
    RLSP volume (so that neighbouring voxels differ) smoothed by the oracle
    with the reference's FP32 sum and quotient equals the kernel's smoothed
    WET at every voxel, the grid's edges included.  A single sample taken
    from another voxel would change the bits.  Beams along the image axes
    put samples exactly on half-voxels (2, 3 and 1 mm; 3 mm is not a power
    of two, so the quotient is formed by division there)."""
    import ctypes
    from dosecuda_b200 import _lib
    case = pkg[2].heterogeneous(13, (gantry,), 40, shape=(37, 45, 51), spacing=spacing,
                                n_slabs=1, n_spheres=1, semi_range=(4.0 * spacing, 5.0 * spacing),
                                centre_jitter=3.0 * spacing, body_inset=5.0 * spacing)
    beam = case.plan.beam_list[0]
    beam.couch_angle = couch
    g = case.grid
    dp = g.prepareIMPTPlan(case.plan, 0, wet_mode="exact")
    rng = np.random.default_rng(int(gantry * 10 + couch))
    rlsp = torch.from_numpy(rng.uniform(0.0, 2.5, g.HU.size).astype(np.float32)).to(DEV)
    raw = torch.empty_like(dp.wet)
    wet = torch.empty_like(dp.wet)
    _lib.check(_lib.lib.pb_wet(_lib.ptr(rlsp), 0, ctypes.byref(dp.grid),
                               ctypes.cast(dp.geoms, ctypes.c_void_p), dp.n_beams, _lib.ptr(raw),
                               _lib.ptr(wet), None,
                               ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)))
    torch.cuda.synchronize(DEV)
    _, ob, _, _ = _oracle_beam(oracle, g, beam, _model(case.plan, beam))
    raw_np = raw.cpu().numpy().reshape(g.HU.shape)
    want = oracle.smooth_f32(raw_np, g.spacing[0], ob)
    got = wet.cpu().numpy().reshape(g.HU.shape)
    assert (raw_np * 10.0 > 9.0).mean() > 0.5   # most voxels take all nine radii
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_pencil_beam_pass_matches_reference_same_wet(pkg, small, curve, reference_module):
    engine = pkg[1]
    g, plan = small.grid, small.plan
    rw, rd = _reference_plan(reference_module, small, curve)
    for b, beam in enumerate(plan.beam_list):
        dp = engine.DevicePlan(g.HU.shape, float(g.spacing[0]), np.asarray(g.origin, np.float32),
                               [engine.BeamSpec(beam.gantry_angle, beam.couch_angle, beam.iso,
                                                beam.spot_list, _model(plan, beam))], DEV)
        dp.set_wet(torch.from_numpy(rw[b]).to(DEV))
        assert max_rel(dp.forward().cpu().numpy().reshape(g.HU.shape), rd[b]) <= 2e-4


def test_dose_kernels_dropin_matches_reference(pkg, small, curve, reference_module):
    from dosecuda_b200 import dose_kernels as mine
    g, plan = small.grid, small.plan
    rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
    for beam in plan.beam_list:
        model = _model(plan, beam)
        beam.spot_list = np.asarray(beam.spot_list, np.float32).reshape(-1, 4)
        w_ref = reference_module.proton_raytrace_cuda(model, _vol(rlsp, g), beam, 0)
        w_mine = mine.proton_raytrace_cuda(model, _vol(rlsp, g), beam, 0)
        assert w_mine.dtype == np.float32 and w_mine.shape == w_ref.shape
        # every voxel, as the other texture-mode tests (ties included)
        assert np.abs(w_mine - w_ref).max() <= 1e-4
        d_ref = reference_module.proton_spot_cuda(model, _vol(rlsp, g), _vol(w_ref, g), beam, 0)
        d_mine = mine.proton_spot_cuda(model, _vol(rlsp, g), _vol(w_ref, g), beam, 0)
        assert max_rel(d_mine, d_ref) <= 2e-4


def test_compute_plan_matches_reference_loop(pkg, small, curve, reference_module):
    g, plan = small.grid, small.plan
    plan.n_fractions = 3
    try:
        g.computeIMPTPlan(plan, 0)
        rw, rd = _reference_plan(reference_module, small, curve)
        want = np.zeros(g.HU.shape, np.float32)
        for d in rd:
            want += d
        want *= plan.n_fractions
        assert g.dose.shape == g.HU.shape and g.dose.dtype == np.float32
        assert max_rel(g.dose, want) <= 1e-3
        for b, d in enumerate(rd):
            assert max_rel(g.beam_doses[b], d * plan.n_fractions) <= 1e-3
        assert np.array_equal(g.RLSP, np.array(np.interp(g.HU, *curve), dtype=np.single))
    finally:
        plan.n_fractions = 1


def test_negative_energy_id_gives_zero_dose_like_reference(pkg, small, curve):
    """A negative energy id sorts first and blocks every layer in importLayers
    (IMPTClasses.cu:37-67): the reference returns a zero dose."""
    from dosecuda_b200 import dose_kernels as mine
    g, plan = small.grid, small.plan
    beam = plan.beam_list[0]
    sl = np.array(beam.spot_list, np.float32).reshape(-1, 4).copy()
    sl[0, 3] = -1.0
    from dosecuda_b200.plan_impt import IMPTBeam
    b2 = IMPTBeam(beam)
    b2.spot_list = sl
    rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
    w = np.ones(g.HU.shape, np.float32)
    d_mine = mine.proton_spot_cuda(_model(plan, beam), _vol(rlsp, g), _vol(w, g), b2, 0)
    assert not d_mine.any()


# -------------------------------------------------------------- gradient

def test_adjoint_matches_oracle(pkg, small, oracle):
    g, plan = small.grid, small.plan
    dp = g.prepareIMPTPlan(plan, 0, wet_mode="exact")
    shape = g.HU.shape
    w = np.random.default_rng(1).normal(size=shape).astype(np.float32)
    got = dp.adjoint(torch.from_numpy(w.reshape(-1)).to(DEV)).cpu().numpy()
    wet = dp.wet.cpu().numpy().reshape(dp.n_beams, *shape)
    want = []
    for b, beam in enumerate(plan.beam_list):
        m, ob, spots, layers = _oracle_beam(oracle, g, beam, _model(plan, beam))
        want.append(oracle.adjoint(wet[b], g.spacing[0], ob, m, spots, layers,
                                   w.astype(np.float64)))
    want = np.concatenate(want)
    assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()


def test_gradient_central_differences(pkg, small, oracle):
    """d(objective)/d(mu) from the adjoint kernel vs FP64 central differences
    of the oracle objective on 200 seeded spots."""
    g, plan = small.grid, small.plan
    presc, wts = small.presc, small.weights
    obj, grad = g.computeIMPTPlanGradient(plan, presc, wts, 0, wet_mode="exact")
    dp = g.prepareIMPTPlan(plan, 0, wet_mode="exact")
    shape = g.HU.shape
    wet = dp.wet.cpu().numpy().reshape(dp.n_beams, *shape)
    # FP64 oracle dose and single-spot columns (dose is linear in mu)
    D = np.zeros(shape)
    cols = []  # (plan row, beam, sorted index)
    per_beam = []
    for b, beam in enumerate(plan.beam_list):
        m, ob, spots, layers = _oracle_beam(oracle, g, beam, _model(plan, beam))
        D += oracle.dose(wet[b], g.spacing[0], ob, m, spots, layers)
        per_beam.append((m, ob, np.asarray(beam.spot_list, np.float32).reshape(-1, 4)))
    nrow = [len(pb[2]) for pb in per_beam]
    rng = np.random.default_rng(42)
    picks = rng.choice(sum(nrow), size=min(200, sum(nrow)), replace=False)
    offs = np.cumsum([0] + nrow)
    presc64 = presc.astype(np.float64)
    w64 = wts.astype(np.float64)

    def objective(Dv):
        return float(np.sum(w64 * (Dv - presc64) ** 2))

    fd = []
    for p in picks:
        b = int(np.searchsorted(offs, p, side="right") - 1)
        row = int(p - offs[b])
        m, ob, sl = per_beam[b]
        one = sl[row:row + 1].copy()
        mu = float(one[0, 2])
        one[0, 2] = 1.0
        spots, layers = oracle.build_layers(one, m.dvp)
        col = oracle.dose(wet[b], g.spacing[0], ob, m, spots, layers)
        h = 1e-3 * max(abs(mu), 1.0)
        fd.append((objective(D + h * col) - objective(D - h * col)) / (2 * h))
    fd = np.array(fd)
    err = np.abs(grad[picks] - fd)
    assert err.max() <= 1e-3 * np.abs(fd).max()
    assert abs(obj - objective(D)) <= 1e-4 * objective(D)


def test_position_gradient_central_differences(pkg, small, oracle):
    """d/dx and d/dy of sum_v w_v D_v with respect to the spot positions
    (pb_dose_adjoint_positions) against FP64 central differences of the
    oracle's single-spot doses on 40 seeded spots (h = 0.05 mm, the float
    step measured), with the weight gradient of the same call against the
    oracle adjoint."""
    g, plan = small.grid, small.plan
    dp = g.prepareIMPTPlan(plan, 0, wet_mode="exact")
    shape = g.HU.shape
    wet = dp.wet.cpu().numpy().reshape(dp.n_beams, *shape)
    w = np.random.default_rng(5).normal(size=shape)
    gw, gx, gy = dp.adjoint_positions(torch.from_numpy(w.reshape(-1).astype(np.float32)).to(DEV))
    gx = dp.to_plan(gx).cpu().numpy()
    gy = dp.to_plan(gy).cpu().numpy()
    per_beam, nrow = [], []
    for b, beam in enumerate(plan.beam_list):
        m, ob, spots, layers = _oracle_beam(oracle, g, beam, _model(plan, beam))
        sl = np.asarray(beam.spot_list, np.float32).reshape(-1, 4)
        per_beam.append((m, ob, sl))
        nrow.append(len(sl))
    offs = np.cumsum([0] + nrow)
    picks = np.random.default_rng(11).choice(offs[-1], size=40, replace=False)
    fdx, fdy = [], []
    for p in picks:
        b = int(np.searchsorted(offs, p, side="right") - 1)
        row = int(p - offs[b])
        m, ob, sl = per_beam[b]
        out = []
        for axis in (0, 1):
            cols = []
            for sign in (1.0, -1.0):
                one = sl[row:row + 1].copy()
                one[0, axis] = np.float32(one[0, axis] + sign * 0.05)
                spots, layers = oracle.build_layers(one, m.dvp)
                cols.append((float(one[0, axis]),
                             oracle.dose(wet[b], g.spacing[0], ob, m, spots, layers)))
            (xp, dpos), (xm, dneg) = cols
            out.append(float(np.sum(w * (dpos - dneg))) / (xp - xm))
        fdx.append(out[0])
        fdy.append(out[1])
    fdx, fdy = np.array(fdx), np.array(fdy)
    scale = max(np.abs(fdx).max(), np.abs(fdy).max())
    assert np.abs(gx[picks] - fdx).max() <= 2e-3 * scale
    assert np.abs(gy[picks] - fdy).max() <= 2e-3 * scale
    g_ref = dp.adjoint(torch.from_numpy(w.reshape(-1).astype(np.float32)).to(DEV))
    assert torch.allclose(gw, g_ref, rtol=1e-5, atol=1e-6 * float(g_ref.abs().max()))


def test_autograd_backward_is_adjoint(pkg, small):
    from dosecuda_b200 import autograd
    g, plan = small.grid, small.plan
    dp = g.prepareIMPTPlan(plan, 0)
    mu = dp.mu_plan().clone().requires_grad_(True)
    presc = torch.from_numpy(small.presc.reshape(-1)).to(DEV)
    w = torch.from_numpy(small.weights.reshape(-1)).to(DEV)
    d = autograd.dose(mu, dp)
    obj = autograd.quadratic_objective(d, presc, w)
    obj.backward()
    o2, g2 = autograd.plan_objective_and_grad(dp, small.presc, small.weights)
    assert abs(float(obj.detach()) - o2) <= 1e-9 * abs(o2)
    # the adjoint's cross-tile sums use float atomics: equal up to rounding
    assert np.allclose(mu.grad.cpu().numpy(), g2, rtol=1e-5, atol=1e-5 * np.abs(g2).max())
    d64 = d.detach().double()
    want = float(torch.sum(w.double() * (d64 - presc.double()) ** 2))
    assert abs(float(obj.detach()) - want) <= 1e-9 * want


# ----------------------------------------------- full-size properties

def test_full_size_linearity_additivity_determinism(pkg):
    phantoms = pkg[2]
    case = phantoms.config_forward_heterogeneous()
    dp = case.grid.prepareIMPTPlan(case.plan, 0)
    d1, bd = dp.forward(beam_doses=True)
    d1b = dp.forward()
    assert torch.equal(d1, d1b)                                  # deterministic
    d2 = dp.forward(dp.mu_sorted * 2.0)
    assert torch.allclose(d2, 2.0 * d1, rtol=1e-5, atol=1e-6 * float(d1.max()))  # linear in mu
    assert torch.allclose(bd.sum(0), d1, rtol=1e-5, atol=1e-6 * float(d1.max()))  # beams add up
    assert float(d1.max()) > 0


def test_full_size_sampled_voxels_vs_oracle(pkg, oracle, curve):
    """Heterogeneous 256x256x160 plan: raw WET, smoothed WET and dose at
    sampled voxels (the hottest and a random set) against the oracle."""
    phantoms = pkg[2]
    case = phantoms.config_forward_heterogeneous()
    g, plan = case.grid, case.plan
    dp = g.prepareIMPTPlan(plan, 0, wet_mode="exact")
    dose = dp.forward().cpu().numpy()
    wet = dp.wet.cpu().numpy()
    raw = dp.raw_wet.cpu().numpy()
    rng = np.random.default_rng(3)
    idx = np.unique(np.concatenate([np.argsort(dose)[-400:],
                                    rng.choice(dose.size, 600, replace=False)])).astype(np.int64)
    rlsp = oracle.rlsp_from_hu(g.HU, *curve)
    want = np.zeros(len(idx))
    for b, beam in enumerate(plan.beam_list):
        m, ob, spots, layers = _oracle_beam(oracle, g, beam, _model(plan, beam))
        raw_o = oracle.raytrace(rlsp, g.spacing[0], ob, idx)
        assert np.abs(raw[b][idx] - raw_o).max() <= 1e-4
        sm_o = oracle.smooth(raw[b].reshape(g.HU.shape), g.spacing[0], ob, idx)
        assert np.abs(wet[b][idx] - sm_o).max() <= 1e-4
        want += oracle.dose(wet[b].reshape(g.HU.shape), g.spacing[0], ob, m, spots, layers, idx)
    assert np.abs(dose[idx] - want).max() <= 2e-4 * dose.max()


def _without_layer_bounds(dp):
    """A copy of dp's device layer records with bound_ok cleared."""
    words = dp.layers.view(torch.int32).reshape(-1, 12).clone()
    words[:, 11] = 0
    return words.view(torch.uint8).reshape(-1)


@pytest.mark.parametrize("which", ["small", "full"])
def test_layer_bounds_change_no_result(pkg, small, which):
    """The per-(tile, layer) skip from pb_layer_bounds drops only layers the
    per-spot cull would empty: dose, per-beam dose and gradient are
    bit-identical with the bounds cleared."""
    phantoms = pkg[2]
    case = small if which == "small" else phantoms.config_gradient()
    dp = case.grid.prepareIMPTPlan(case.plan, 0)
    words = dp.layers.view(torch.int32).reshape(-1, 12)
    assert int(words[:, 11].min()) == 1          # every layer got its bounds
    presc, wts = case.objective_fields()
    d1, bd1 = dp.forward(beam_doses=True)
    from dosecuda_b200 import engine
    resid = torch.empty_like(d1)
    engine.objective(d1, torch.from_numpy(presc.reshape(-1)).to(DEV),
                     torch.from_numpy(wts.reshape(-1)).to(DEV), resid)
    g1 = dp.adjoint(resid).clone()
    n1 = dp.count_evaluated()
    bounded = dp.layers
    dp.layers = _without_layer_bounds(dp)
    try:
        d2, bd2 = dp.forward(beam_doses=True)
        g2 = dp.adjoint(resid)
        n2 = dp.count_evaluated()
    finally:
        dp.layers = bounded
    assert torch.equal(d1, d2) and torch.equal(bd1, bd2)
    # the same spots survive the cull: the same exp2 and evaluation counts
    assert n1 == n2 and n1[1] <= n1[0] <= 2 * n1[1] and n1[1] > 0
    # the adjoint sums tile partials with float atomics in any order
    assert torch.allclose(g1, g2, rtol=1e-5, atol=1e-6 * float(g1.abs().max()))


@pytest.mark.parametrize("which", ["small", "full"])
def test_tile_order_is_a_permutation_and_changes_no_result(pkg, small, which):
    """pb_tile_order: every tile of the default shape once, the estimated
    most expensive first; pb_dose_ordered gives pb_dose's dose and per-beam
    doses bit for bit, pb_dose_adjoint_ordered its gradient to float
    rounding (atomic order)."""
    import ctypes
    from dosecuda_b200 import _lib
    case = small if which == "small" else pkg[2].config_gradient()
    dp = case.grid.prepareIMPTPlan(case.plan, 0)
    order = dp.tile_order().cpu().numpy()
    n = int(_lib.lib.pb_tile_order_count(ctypes.byref(dp.grid)))
    assert order.shape == (n,) and np.array_equal(np.sort(order), np.arange(n))
    st = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    d0 = torch.empty(dp.n_vox, device=DEV)
    b0 = torch.empty((dp.n_beams, dp.n_vox), device=DEV)
    _lib.check(_lib.lib.pb_dose(ctypes.byref(dp.grid), ctypes.cast(dp.beams, ctypes.c_void_p),
                                dp.n_beams, _lib.ptr(dp.wet), _lib.ptr(dp.layers),
                                _lib.ptr(dp.spot_geo), _lib.ptr(dp.mu_sorted), 2.0,
                                _lib.ptr(d0), _lib.ptr(b0), st), "pb_dose")
    d1, b1 = dp.forward(scale=2.0, beam_doses=True)
    assert torch.equal(d0, d1) and torch.equal(b0, b1)
    assert torch.equal(dp.forward(), d0 / 2.0)      # scale 2 is exact
    w = torch.from_numpy(np.random.default_rng(5).normal(size=dp.n_vox).astype(np.float32))
    w = w.to(DEV)
    g0 = torch.empty(max(dp.n_spots, 1), device=DEV)
    _lib.check(_lib.lib.pb_dose_adjoint(ctypes.byref(dp.grid),
                                        ctypes.cast(dp.beams, ctypes.c_void_p), dp.n_beams,
                                        _lib.ptr(dp.wet), _lib.ptr(dp.layers),
                                        _lib.ptr(dp.spot_geo), _lib.ptr(w), 1.0, _lib.ptr(g0), st),
               "pb_dose_adjoint")
    g1 = dp.adjoint(w)
    m = float(g0.abs().max())
    assert m > 0 and float((g0[: dp.n_spots] - g1).abs().max()) <= 1e-5 * m


def test_tile_order_on_grids_smaller_than_a_tile(pkg, small):
    """Grids of fewer voxels than one line tile (and fewer tiles than a warp
    of the cost kernel takes): the order still names every tile once and
    the ordered dose equals the unordered one bit for bit."""
    import ctypes
    from dosecuda_b200 import _lib, engine
    beam = small.plan.beam_list[0]
    model = _model(small.plan, beam)
    spots = np.asarray(beam.spot_list, np.float32).reshape(-1, 4)[:40]
    for shape in [(3, 5, 9), (9, 17, 8)]:
        spacing = 3.0
        origin = np.asarray(beam.iso, np.float32) - 0.5 * spacing * np.array(shape[::-1], np.float32)
        dp = engine.DevicePlan(shape, spacing, origin,
                               [engine.BeamSpec(beam.gantry_angle, beam.couch_angle, beam.iso,
                                                spots, model)], DEV)
        dp.compute_wet(torch.ones(int(np.prod(shape)), device=DEV))
        order = dp.tile_order().cpu().numpy()
        n = int(_lib.lib.pb_tile_order_count(ctypes.byref(dp.grid)))
        assert n >= 1 and np.array_equal(np.sort(order[:n]), np.arange(n)), shape
        d0 = torch.empty(dp.n_vox, device=DEV)
        st = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
        _lib.check(_lib.lib.pb_dose(ctypes.byref(dp.grid),
                                    ctypes.cast(dp.beams, ctypes.c_void_p), dp.n_beams,
                                    _lib.ptr(dp.wet), _lib.ptr(dp.layers), _lib.ptr(dp.spot_geo),
                                    _lib.ptr(dp.mu_sorted), 1.0, _lib.ptr(d0), None, st), "pb_dose")
        assert torch.equal(dp.forward(), d0), shape


def test_beam_at_a_time_forward_and_compute_plan(small):
    """forward_beam(b), each beam alone in its own tile order, gives the
    bits of the all-beam launch's per-beam dose; computeIMPTPlan, which
    runs the beams one at a time, returns those doses times n_fractions and
    their float32 sum times n_fractions, as the reference forms them
    (plan_impt.py:201-206)."""
    g, plan = small.grid, small.plan
    dp = g.prepareIMPTPlan(plan, 0)
    _, bd = dp.forward(beam_doses=True)
    for b in range(dp.n_beams):
        order = dp.beam_tile_order(b).cpu()
        assert torch.equal(order.sort().values, torch.arange(order.numel(), dtype=order.dtype))
        assert torch.equal(dp.forward_beam(b), bd[b])
    # the last beam in launches over groups of z slabs of tiles (5 slabs
    # here): each fills exactly its voxel range, together the whole volume
    b = dp.n_beams - 1
    n = dp.beam_tile_order(b).numel()
    for k in (1, 2, 4, 9):
        parts = dp.beam_tile_order_parts(b, k)
        assert len(parts) == min(k, 5) and parts[0][1] == 0 and parts[-1][2] == dp.n_vox
        listed = torch.cat([o[o >= 0] for o, _, _ in parts]).cpu()
        assert torch.equal(listed.sort().values, torch.arange(n, dtype=listed.dtype))
        out = torch.full((dp.n_vox,), float("nan"), device=DEV)
        for o, v0, v1 in parts:
            assert v0 < v1
            dp.forward_beam(b, out=out, order=o)
            assert torch.equal(out[:v1], bd[b, :v1]) and bool(torch.isnan(out[v1:]).all())
    bd = bd.cpu().numpy()
    plan.n_fractions = 3
    try:
        g.computeIMPTPlan(plan, 0)
    finally:
        plan.n_fractions = 1
    want = np.zeros(bd.shape[1], np.float32)
    for b in range(bd.shape[0]):
        assert np.array_equal(g.beam_doses[b].reshape(-1), bd[b] * np.float32(3))
        want += bd[b]
    want *= np.float32(3)
    assert np.array_equal(g.dose.reshape(-1), want)


def test_caller_hu_locked_in_place_on_second_use(pkg):
    """computeIMPTPlan page-locks a caller's float32 HU array in place on its
    second use (pb_host_register) and releases it when the array is
    collected; the results do not change."""
    import gc
    from dosecuda_b200 import plan_impt
    case = pkg[2].small_heterogeneous()
    g, plan = case.grid, case.plan
    hu = np.ascontiguousarray(g.HU, dtype=np.float32).copy()
    g.HU = hu
    key = (hu.ctypes.data, hu.nbytes)
    assert hu.nbytes >= 1 << 18
    g.computeIMPTPlan(plan, 0)
    first = g.dose.copy()
    assert key not in plan_impt._HOST_LOCKED and not torch.from_numpy(hu).is_pinned()
    g.computeIMPTPlan(plan, 0)
    assert key in plan_impt._HOST_LOCKED and torch.from_numpy(hu).is_pinned()
    g.computeIMPTPlan(plan, 0)
    assert np.array_equal(g.dose, first)
    g.HU = hu.copy()
    del hu
    gc.collect()
    assert key not in plan_impt._HOST_LOCKED


def test_adjoint_counts_follow_its_tile_skip(small):
    """pb_count_evaluated_adjoint: on a field nonzero everywhere it counts
    the forward's work; on a zero field nothing; on a field nonzero in one
    slab of z only the tiles that reach the slab, so less than the forward
    and more than nothing."""
    dp = small.grid.prepareIMPTPlan(small.plan, 0)
    fwd = dp.count_evaluated()
    V = dp.n_vox
    assert dp.count_evaluated_adjoint(torch.ones(V, device=DEV)) == fwd
    assert dp.count_evaluated_adjoint(torch.ones(V, device=DEV), scale=2.0) == fwd
    assert dp.count_evaluated_adjoint(torch.zeros(V, device=DEV)) == (0, 0)
    nz = small.grid.HU.shape[0]
    slab = torch.zeros(small.grid.HU.shape, device=DEV)
    slab[nz // 2] = 1.0
    part = dp.count_evaluated_adjoint(slab.reshape(-1))
    assert 0 < part[0] < fwd[0] and 0 < part[1] < fwd[1]


def test_layer_bounds_values(pkg, small):
    """pb_layer_bounds against a host recomputation: spot boxes and the LUT
    row maxima exactly, the halo-sigma bound at least the formula's maximum
    on a dense depth grid."""
    g, plan = small.grid, small.plan
    dp = g.prepareIMPTPlan(plan, 0)
    rec = dp.layers.cpu().numpy().view(pkg[0]._lib.LAYER_DTYPE)
    geo = dp.spot_geo.cpu().numpy()
    for b in range(dp.n_beams):
        t = dp.tables[b]
        sig = t.sigmas.cpu().numpy()
        for l in range(dp.n_layers[b]):
            L = rec[dp.layer_offsets[b] + l]
            s0 = dp.spot_offsets[b] + int(L["spot_start"])
            xy = geo[s0:s0 + int(L["n_spots"]), :2]
            assert L["bound_ok"] == 1
            assert (L["sx0"], L["sx1"]) == (xy[:, 0].min(), xy[:, 0].max())
            assert (L["sy0"], L["sy1"]) == (xy[:, 1].min(), xy[:, 1].max())
            assert L["mcs_max"] == np.abs(sig[int(L["energy_id"])]).max()
            r80 = float(L["r80"])
            hi = float(np.float32(r80) - np.float32(0.1))
            w = np.linspace(min(0.1, hi), hi, 20001)
            a1 = w - r80 - 5.0
            sh = 2.85 + 0.0014 * r80 * np.log(w + 3.0) + 0.06 * w - 7.4e-5 * w * w - \
                (0.22 * r80) / (a1 * a1)
            assert L["sh_max"] >= max(sh.max(), 0.0)
            assert L["sh_max"] <= max(sh.max(), 0.0) + 0.05


def test_count_pairs_matches_oracle(pkg, small, oracle):
    g, plan = small.grid, small.plan
    dp = g.prepareIMPTPlan(plan, 0)
    wet = dp.wet.cpu().numpy().reshape(dp.n_beams, *g.HU.shape)
    want = 0
    for b, beam in enumerate(plan.beam_list):
        _, _, _, layers = _oracle_beam(oracle, g, beam, _model(plan, beam))
        want += oracle.count_pairs(wet[b], layers)
    assert dp.count_pairs() == want


# ------------------------------------------------------------ error paths

def test_invalid_device_raises_runtime_error(pkg, small, curve):
    from dosecuda_b200 import dose_kernels as mine
    g, plan = small.grid, small.plan
    beam = plan.beam_list[0]
    rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
    with pytest.raises(RuntimeError, match="CUDA error"):
        mine.proton_raytrace_cuda(_model(plan, beam), _vol(rlsp, g), beam, 97)


def _one_beam(plan, beam):
    p = plan.__class__.__new__(plan.__class__)
    p.__dict__.update(plan.__dict__)
    p.beam_list = [beam]
    p.n_beams = 1
    return p


def test_edge_plans_empty_and_single_spot_beams(pkg, small):
    """A beam without spots adds nothing (its layers are empty); a beam of
    one spot, added as the reference's addSingleSpot leaves it (a 1-D
    spot_list), gives that spot's dose; a plan whose every beam is empty
    gives zero dose and an empty gradient."""
    from dosecuda_b200.plan_impt import IMPTBeam
    g, plan = small.grid, small.plan
    b0 = plan.beam_list[0]
    empty = IMPTBeam(b0)
    empty.resetSpots()
    single = IMPTBeam(b0)
    single.resetSpots()
    x, y, mu, e = np.asarray(b0.spot_list, np.float32).reshape(-1, 4)[0]
    single.addSingleSpot(x, y, mu, e)
    assert np.asarray(single.spot_list).ndim == 1

    d_ref = g.prepareIMPTPlan(_one_beam(plan, b0), 0).forward()
    two = _one_beam(plan, b0)
    two.beam_list = [b0, empty]
    two.n_beams = 2
    dp2 = g.prepareIMPTPlan(two, 0)
    assert torch.equal(dp2.forward(), d_ref)

    solo = g.prepareIMPTPlan(_one_beam(plan, single), 0)
    full = g.prepareIMPTPlan(_one_beam(plan, b0), 0)
    mu_rows = torch.zeros(full.n_spots, dtype=torch.float32, device=DEV)
    mu_rows[0] = float(mu)               # plan row 0 only
    mu1 = full.to_sorted(mu_rows)
    assert solo.n_spots == 1
    d1 = solo.forward()
    assert float(d1.max()) > 0
    assert torch.allclose(d1, full.forward(mu1), rtol=1e-6, atol=1e-7 * float(d1.max()))

    none = _one_beam(plan, empty)
    dpn = g.prepareIMPTPlan(none, 0)
    assert dpn.n_spots == 0 and float(dpn.forward().abs().max()) == 0.0
    assert dpn.adjoint(torch.ones(dpn.n_vox, dtype=torch.float32, device=DEV)).numel() == 0


def test_plan_with_more_beams_than_one_launch(pkg, curve):
    """18 beams (more than the 16 a launch takes): computeIMPTPlan and
    computeIMPTPlanGradient work in groups; every beam's dose matches the
    same beam alone, the plan dose is their sum, and each group's gradient
    is its adjoint of the whole plan's residual."""
    from dosecuda_b200 import engine
    angles = tuple(float(a) for a in range(0, 360, 20))
    case = pkg[2].heterogeneous(9, angles, 18 * 40, shape=(32, 40, 40), spacing=4.0,
                                n_slabs=1, n_spheres=1, semi_range=(12.0, 16.0),
                                centre_jitter=2.0, body_inset=12.0)
    g, plan = case.grid, case.plan
    assert len(plan.beam_list) == 18
    g.computeIMPTPlan(plan, 0)
    assert len(g.beam_doses) == 18
    total = np.sum(np.stack(g.beam_doses), axis=0, dtype=np.float64)
    assert np.allclose(g.dose, total, rtol=1e-5, atol=1e-6 * total.max())
    for b in (0, 17):
        one = _one_beam(plan, plan.beam_list[b])
        d = g.prepareIMPTPlan(one, 0).forward().cpu().numpy().reshape(g.HU.shape)
        assert np.allclose(g.beam_doses[b], d, rtol=1e-6, atol=1e-7 * d.max())
    presc, wts = case.objective_fields()
    obj, grad = g.computeIMPTPlanGradient(plan, presc, wts, 0)
    assert grad.shape == (sum(np.asarray(b.spot_list).reshape(-1, 4).shape[0]
                              for b in plan.beam_list),)
    dose = torch.from_numpy(g.dose.reshape(-1)).to(DEV)
    resid = torch.empty_like(dose)
    o_ref = float(engine.objective(dose, torch.from_numpy(presc.reshape(-1)).to(DEV),
                                   torch.from_numpy(wts.reshape(-1)).to(DEV), resid))
    assert abs(obj - o_ref) <= 1e-6 * o_ref
    last = _one_beam(plan, plan.beam_list[17])
    dp = g.prepareIMPTPlan(last, 0)
    g17 = dp.to_plan(dp.adjoint(resid)).cpu().numpy()
    assert np.allclose(grad[-len(g17):], g17, rtol=1e-4, atol=1e-5 * np.abs(g17).max())


def test_ray_cap_status_is_zero_on_valid_geometry(pkg, small):
    dp = small.grid.prepareIMPTPlan(small.plan, 0)
    assert int(dp._status.item()) == 0
