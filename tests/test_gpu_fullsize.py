"""Parity at the benchmarked sizes (256x256x160 at 2 mm and up).

* Texture-mode WET and dose of the 3-beam (~8k spots) and 4-beam (~19k
  spots) heterogeneous plans against the reference's own CUDA module
  (oracle/_ref) at every voxel: dose within 1e-3 of Dmax (the drop-in bar)
  and the WET maximum stated.  The WET residue is the reference's FP32
  running sum (fmaf per 1 mm sample, CudaClasses.cu:206-222) against the
  FP64 sum here, which grows with the ray length.
* The pencil-beam pass alone on the reference's own WET: within 1e-3 of
  Dmax at every voxel, and at the 40 voxels where it differs most from the
  reference, within 2e-5 of Dmax of the FP64 oracle on that WET.  At full
  size the reference's FP32 axis distance |ray|^2 - (t.ray)^2/|t|^2
  (IMPTClasses.cu:123-133) loses digits to cancellation (both terms are
  ~Z^2 at depth); this path forms |t x ray|^2/|t|^2, which does not.
* The 4-beam plan's spot-weight gradient (texture WET, the benchmarked
  step) against the FP64 oracle adjoint on 200 seeded spots, same WET and
  residual: within 1e-4 of max |g| over those spots.
* The 32-plan batch of the batched benchmark (grids up to 200x200x160,
  1-4 beams, 500-20,000 spots) against each plan computed alone: equal bit
  for bit (same kernel shape), also after a CUDA-graph replay.
* The 512x512x200 optimisation loop (~60k spots): the final dose after
  projected-gradient iterations against the FP64 oracle at the 400 hottest
  and 600 random voxels, on the same WET and weights: within 1e-4 of Dmax.
"""
import numpy as np
import pytest
import torch

from conftest import cuda_available, max_rel

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DEV = torch.device("cuda", 0)


def _model(plan, beam):
    labels = list(plan.dicom_rangeshifter_label.astype(str))
    return plan.beam_models[labels.index(beam.dicom_rangeshifter_label)]


def _vol(data, grid):
    from dosecuda_b200.plan import VolumeObject
    v = VolumeObject()
    v.voxel_data = np.ascontiguousarray(data, np.float32)
    v.origin = np.array(grid.origin, np.float32)
    v.spacing = np.array(grid.spacing, np.float32)
    return v


@pytest.fixture(scope="module")
def curve():
    from dosecuda_b200.plan_impt import _hu_curve
    return _hu_curve("HitachiProbeatJHU")


@pytest.mark.parametrize("which", ["three_beams_8k", "four_beams_20k"])
def test_full_size_texture_mode_matches_reference_every_voxel(which, curve, reference_module,
                                                               oracle):
    from dosecuda_b200 import engine, phantoms
    case = (phantoms.config_forward_heterogeneous() if which == "three_beams_8k"
            else phantoms.config_gradient())
    g, plan = case.grid, case.plan
    shape = g.HU.shape
    dp = g.prepareIMPTPlan(plan, 0, wet_mode="texture")
    assert int(dp._status.item()) == 0
    wet = dp.wet.cpu().numpy().reshape(dp.n_beams, *shape)
    dose, bd = dp.forward(beam_doses=True)
    dose = dose.cpu().numpy().reshape(shape)
    bd = bd.cpu().numpy().reshape(dp.n_beams, *shape)

    rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
    ref_total = np.zeros(shape, np.float64)
    dwet, dbeam, dpass, dor_mine, dor_ref = [], [], [], [], []
    for b, beam in enumerate(plan.beam_list):
        model = _model(plan, beam)
        beam.spot_list = np.asarray(beam.spot_list, np.float32).reshape(-1, 4)
        rw = reference_module.proton_raytrace_cuda(model, _vol(rlsp, g), beam, 0)
        rd = reference_module.proton_spot_cuda(model, _vol(rlsp, g), _vol(rw, g), beam, 0)
        ref_total += rd
        dwet.append(float(np.abs(wet[b] - rw).max()))
        dbeam.append(max_rel(bd[b], rd))
        # this path's pencil-beam pass on the reference's own WET
        one = engine.DevicePlan(shape, float(g.spacing[0]), np.asarray(g.origin, np.float32),
                                [engine.BeamSpec(beam.gantry_angle, beam.couch_angle, beam.iso,
                                                 beam.spot_list, model)], DEV)
        one.set_wet(torch.from_numpy(rw).to(DEV))
        mine = one.forward().cpu().numpy().reshape(shape)
        dpass.append(max_rel(mine, rd))
        del one
        # the FP64 oracle on the reference's WET where the two differ most
        idx = np.argsort(np.abs(mine - rd).ravel())[-40:].astype(np.int64)
        m = oracle.Model(model)
        ob = oracle.beam_setup(beam.gantry_angle, beam.couch_angle, m.vsadx, m.vsady,
                               beam.iso, g.origin)
        spots, lay = oracle.build_layers(beam.spot_list, m.dvp)
        want = oracle.dose(rw, g.spacing[0], ob, m, spots, lay, idx)
        dmax = float(rd.max())
        dor_mine.append(float(np.abs(mine.ravel()[idx] - want).max() / dmax))
        dor_ref.append(float(np.abs(rd.ravel()[idx] - want).max() / dmax))
    dtot = max_rel(dose, ref_total)
    print(f"\n{which}: max |dWET| per beam (cm) {dwet}; beam dose err / Dmax {dbeam}; "
          f"pass on reference WET {dpass}; plan dose err / Dmax {dtot:.2e}; "
          f"at the worst voxels vs FP64 oracle: this path {dor_mine}, reference {dor_ref}")
    assert dtot <= 1e-3
    assert max(dbeam) <= 1e-3
    assert max(dpass) <= 1e-3
    assert max(dor_mine) <= 2e-5
    # FP32 running sum (reference) against FP64 (here) over rays of up to
    # ~700 samples: a few 1e-4 cm; a sample from a wrong cell shows as >= 1e-2
    assert max(dwet) <= 1e-3


def test_full_size_gradient_matches_fp64_oracle_adjoint(oracle):
    from dosecuda_b200 import engine, phantoms
    case = phantoms.config_gradient()
    g, plan = case.grid, case.plan
    shape = g.HU.shape
    dp = g.prepareIMPTPlan(plan, 0, wet_mode="texture")
    dose = dp.forward()
    resid = torch.empty_like(dose)
    engine.objective(dose, torch.from_numpy(case.presc.reshape(-1)).to(DEV),
                     torch.from_numpy(case.weights.reshape(-1)).to(DEV), resid)
    grad = dp.to_plan(dp.adjoint(resid)).cpu().numpy()
    wet = dp.wet.cpu().numpy().reshape(dp.n_beams, *shape)
    w64 = resid.cpu().numpy().astype(np.float64)

    rows = [np.asarray(b.spot_list, np.float32).reshape(-1, 4) for b in plan.beam_list]
    offs = np.cumsum([0] + [len(r) for r in rows])
    picks = np.sort(np.random.default_rng(42).choice(offs[-1], size=200, replace=False))
    got, want = [], []
    for b, beam in enumerate(plan.beam_list):
        mine = picks[(picks >= offs[b]) & (picks < offs[b + 1])] - offs[b]
        if len(mine) == 0:
            continue
        # energy order, stable: the oracle's layer build keeps this order
        sub = rows[b][mine]
        order = np.argsort(sub[:, 3], kind="stable")
        sub, mine = sub[order], mine[order]
        m = oracle.Model(_model(plan, beam))
        ob = oracle.beam_setup(beam.gantry_angle, beam.couch_angle, m.vsadx, m.vsady, beam.iso,
                               g.origin)
        spots, layers = oracle.build_layers(sub, m.dvp)
        assert np.array_equal(spots["x"], sub[:, 0]) and np.array_equal(spots["y"], sub[:, 1])
        want.append(oracle.adjoint(wet[b], g.spacing[0], ob, m, spots, layers, w64))
        got.append(grad[offs[b] + mine])
    got, want = np.concatenate(got), np.concatenate(want)
    err = float(np.abs(got - want).max() / np.abs(want).max())
    print(f"\ngradient vs FP64 oracle adjoint, 200 spots: max err / max|g| {err:.2e}")
    assert err <= 1e-4


def test_batch_of_32_uneven_plans_matches_single_plans():
    from dosecuda_b200 import batch, phantoms
    cases = phantoms.batch_cases(seed=4, n_plans=32)   # the batched benchmark's plans
    bp = batch.from_cases(cases, 0)
    assert bp.n_plans == 32 and max(dp.n_vox for dp in bp.plans) >= 150 * 150 * 120
    single_wet = [dp.wet.clone() for dp in bp.plans]
    single = [dp.forward_variant(bp.variant) for dp in bp.plans]
    for dp in bp.plans:
        dp.wet.zero_()
    bp.run()
    torch.cuda.synchronize()
    assert int(bp.status.item()) == 0
    for p, dp in enumerate(bp.plans):
        assert torch.equal(dp.wet, single_wet[p]), p
        assert torch.equal(bp.doses[p], single[p]), p
        assert float(single[p].max()) > 0
    graph = bp.capture()
    for d in bp.doses:
        d.zero_()
    graph.replay()
    torch.cuda.synchronize()
    for p in range(bp.n_plans):
        assert torch.equal(bp.doses[p], single[p]), p


def test_optimisation_loop_512x512x200_final_dose_vs_fp64_oracle(oracle):
    from dosecuda_b200 import optimize, phantoms
    case = phantoms.config_optimisation()
    g, plan = case.grid, case.plan
    assert 55000 <= case.n_spots <= 65000
    dp = g.prepareIMPTPlan(plan, 0)
    opt = optimize.ProjectedGradient(dp, torch.from_numpy(case.presc),
                                     torch.from_numpy(case.weights),
                                     scale=float(plan.n_fractions))
    opt.prepare()
    hist = opt.run(5).cpu().numpy()
    assert np.all(np.diff(hist) <= 1e-9 * hist[0])
    dose = opt.final_dose().cpu().numpy()
    wet = dp.wet.cpu().numpy()
    mu = opt.mu_plan().cpu().numpy()
    rng = np.random.default_rng(0)
    idx = np.unique(np.concatenate([np.argsort(dose)[-400:],
                                    rng.choice(dose.size, 600, replace=False)])).astype(np.int64)
    want = np.zeros(len(idx))
    row = 0
    for b, beam in enumerate(plan.beam_list):
        sl = np.asarray(beam.spot_list, np.float32).reshape(-1, 4).copy()
        sl[:, 2] = mu[row: row + len(sl)]
        row += len(sl)
        m = oracle.Model(_model(plan, beam))
        ob = oracle.beam_setup(beam.gantry_angle, beam.couch_angle, m.vsadx, m.vsady, beam.iso,
                               g.origin)
        spots, layers = oracle.build_layers(sl, m.dvp)
        want += oracle.dose(wet[b].reshape(g.HU.shape), g.spacing[0], ob, m, spots, layers, idx)
    want *= float(plan.n_fractions)
    err = float(np.abs(dose[idx] - want).max() / dose.max())
    print(f"\noptimisation loop final dose vs FP64 oracle, {len(idx)} voxels: {err:.2e} of Dmax")
    assert err <= 1e-4


@pytest.mark.parametrize("gantry,couch", [(120.0, 0.0), (240.0, 0.0), (33.0, 20.0),
                                          (300.0, 90.0)])
def test_full_size_oblique_beams_smoothing_matches_reference(gantry, couch, reference_module):
    """Texture-mode WET of a full 256x256x160 water volume against the
    reference module at every voxel, for oblique and couch-rotated beams.
    Their half-voxel smoothing ties are decided by the last bits of the
    reference's compiled rotations and directions (fused multiply-adds,
    CUDA's sincosf), which the smoothing kernel reproduces; one tie taken the
    other way moves a voxel's WET by ~4e-3 cm here."""
    from dosecuda_b200 import engine, phantoms
    from dosecuda_b200.plan_impt import IMPTBeam
    case = phantoms.config_forward_heterogeneous()
    g, plan = case.grid, case.plan
    shape = g.HU.shape
    water = np.full(shape, np.float32(1.00653), np.float32)
    beam = IMPTBeam(plan.beam_list[0])
    beam.gantry_angle, beam.couch_angle = gantry, couch
    beam.spot_list = np.asarray(plan.beam_list[0].spot_list, np.float32).reshape(-1, 4)
    model = _model(plan, beam)
    dp = engine.DevicePlan(shape, float(g.spacing[0]), np.asarray(g.origin, np.float32),
                           [engine.BeamSpec(gantry, couch, beam.iso, beam.spot_list, model)], DEV)
    dp.compute_wet(torch.from_numpy(water.reshape(-1)).to(DEV))
    wet = dp.wet.cpu().numpy().reshape(shape)
    want = reference_module.proton_raytrace_cuda(model, _vol(water, g), beam, 0)
    d = np.abs(wet - want)
    print(f"\ngantry {gantry} couch {couch}: max |dWET| {d.max():.2e} cm, "
          f"voxels > 1e-3 cm: {int((d > 1e-3).sum())}")
    # the FP32 (reference) against FP64 (here) running sum over rays of up to
    # ~600 samples
    assert d.max() <= 1e-3
