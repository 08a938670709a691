"""The split WET / dose API and the range-shifter model RS4 on the GPU.

* computeIMPTWET, computeIMPTPlanFromWET and writeWETNRRD
  (DoseCUDA/plan_impt.py:208-288) against the reference's own calls
  (oracle/_ref) on the same inputs: WET within 1e-4 cm at every voxel, dose
  on the reference's WET within 2e-4 of Dmax; the NRRD files hold
  computeIMPTWET's volumes bit for bit; a plan dose from the split API equals
  computeIMPTPlan's.
* The RS4 golden case (couch 90 deg, gantry 45 deg, energies whose R80 is
  -0.65 to 13.6 mm, so the halo depth clamp [0.1, R80 - 0.1] of
  IMPTClasses.cu:104-121 is crossed) through the CUDA kernels: the
  texture-mode WET against the reference's WET stored in the fixture
  (1e-4 cm), the pencil-beam pass on that WET against the reference's dose
  (2e-4 of Dmax), the whole chain (1e-3 of Dmax), and the adjoint against
  the FP64 oracle adjoint (1e-4 of max |g|).
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, cuda_available, max_rel

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


@pytest.fixture(scope="module")
def small():
    from dosecuda_b200 import phantoms
    c = phantoms.small_heterogeneous()
    for b in c.plan.beam_list:
        b.spot_list = np.asarray(b.spot_list, np.float32).reshape(-1, 4)
    return c


def test_compute_wet_matches_reference_calls(small, curve, reference_module):
    g, plan = small.grid, small.plan
    wets = g.computeIMPTWET(plan, 0)
    assert len(wets) == len(plan.beam_list)
    rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
    assert np.array_equal(g.RLSP, rlsp)
    for w, beam in zip(wets, plan.beam_list):
        assert w.voxel_data.dtype == np.float32 and w.voxel_data.shape == g.HU.shape
        assert np.array_equal(w.origin, np.array(g.origin, np.float32))
        assert np.array_equal(w.spacing, np.array(g.spacing, np.float32))
        want = reference_module.proton_raytrace_cuda(_model(plan, beam), _vol(rlsp, g), beam, 0)
        assert np.abs(w.voxel_data - want).max() <= 1e-4


def test_plan_from_wet_matches_reference_and_compute_plan(small, curve, reference_module):
    g, plan = small.grid, small.plan
    rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
    plan.n_fractions = 2
    try:
        g.computeIMPTPlan(plan, 0)
        total = np.zeros(g.HU.shape, np.float32)
        for b, (w, beam) in enumerate(zip(g.computeIMPTWET(plan, 0), plan.beam_list)):
            mine = g.computeIMPTPlanFromWET(plan, w, beam, 0)
            assert mine.dtype == np.float32 and mine.shape == g.HU.shape
            total += mine
            # the reference's dose on the same (this path's) WET volume
            want = reference_module.proton_spot_cuda(_model(plan, beam), _vol(rlsp, g), w,
                                                     beam, 0)
            assert max_rel(mine, want) <= 2e-4
            # computeIMPTPlan's per-beam dose carries n_fractions (plan_impt.py:203)
            assert max_rel(g.beam_doses[b], mine * plan.n_fractions) <= 1e-6
        assert max_rel(g.dose, total * plan.n_fractions) <= 1e-6
    finally:
        plan.n_fractions = 1


def test_write_wet_nrrd_holds_compute_wet(small, tmp_path):
    from dosecuda_b200 import nrrd
    g, plan = small.grid, small.plan
    path = str(tmp_path / "wet.nrrd")
    g.writeWETNRRD(plan, path, 0)
    wets = g.computeIMPTWET(plan, 0)
    for i, w in enumerate(wets):
        vol, origin, spacing = nrrd.read(path.replace(".nrrd", "_beam%02i.nrrd" % (i + 1)))
        assert np.array_equal(vol, w.voxel_data)
        assert np.allclose(origin, g.origin) and np.allclose(spacing, g.spacing)
    with pytest.raises(Exception, match="nrrd extension"):
        g.writeWETNRRD(plan, str(tmp_path / "wet.mha"), 0)


# ------------------------------------------------------------------- RS4

def _golden_case(name):
    from dosecuda_b200 import phantoms
    from dosecuda_b200.plan_impt import IMPTBeam, IMPTDoseGrid
    z = np.load(os.path.join(GOLDEN, name))
    g = IMPTDoseGrid()
    g.HU = np.asarray(z["hu"], np.float32)
    g.origin = np.asarray(z["origin"], np.float64)
    g.spacing = np.asarray(z["spacing"], np.float64)
    g.size = np.array(g.HU.shape)
    plan = phantoms._new_plan()
    for b in range(int(z["n_beams"])):
        beam = IMPTBeam()
        beam.gantry_angle = float(z[f"b{b}_gantry"])
        beam.couch_angle = float(z[f"b{b}_couch"])
        beam.iso = np.asarray(z[f"b{b}_iso"], np.float32)
        beam.dicom_rangeshifter_label = str(z[f"b{b}_label"])
        beam.spot_list = np.asarray(z[f"b{b}_spots"], np.float32)
        beam.n_spots = len(beam.spot_list)
        plan.addBeam(beam)
    return z, g, plan


def test_rs4_beam_through_the_kernels_matches_reference_and_oracle(oracle, curve):
    z, g, plan = _golden_case("couch90_rs4.npz")
    beam = plan.beam_list[0]
    assert beam.dicom_rangeshifter_label == "4" and beam.couch_angle == 90.0
    model = _model(plan, beam)
    r80 = model.divergence_params[beam.spot_list[:, 3].astype(int), 1]
    assert r80.min() < 0.2           # the halo depth clamp's bounds cross
    shape = g.HU.shape
    ref_wet, ref_dose = z["b0_wet"], z["b0_dose"]

    dp = g.prepareIMPTPlan(plan, 0, wet_mode="texture")
    wet = dp.wet.cpu().numpy().reshape(shape)
    assert np.abs(wet - ref_wet).max() <= 1e-4
    assert max_rel(dp.forward().cpu().numpy().reshape(shape), ref_dose) <= 1e-3

    # the pencil-beam pass alone, on the reference's own WET
    dp.set_wet(torch.from_numpy(ref_wet).to(DEV))
    assert max_rel(dp.forward().cpu().numpy().reshape(shape), ref_dose) <= 2e-4

    # the adjoint on the same WET against the FP64 oracle adjoint
    w = np.random.default_rng(3).normal(size=shape).astype(np.float32)
    got = dp.adjoint(torch.from_numpy(w.reshape(-1)).to(DEV)).cpu().numpy()
    m = oracle.Model(model)
    ob = oracle.beam_setup(beam.gantry_angle, beam.couch_angle, m.vsadx, m.vsady, beam.iso,
                           g.origin)
    spots, layers = oracle.build_layers(beam.spot_list, m.dvp)
    want = oracle.adjoint(ref_wet, g.spacing[0], ob, m, spots, layers, w.astype(np.float64))
    assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()

    # exact mode, whole chain, against the FP64 oracle
    dpe = g.prepareIMPTPlan(plan, 0, wet_mode="exact")
    want_d = oracle.plan_forward(g.HU, g.origin, g.spacing[0],
                                 [(beam.gantry_angle, beam.couch_angle, beam.iso,
                                   beam.spot_list, model)],
                                 curve)["dose"]
    assert max_rel(dpe.forward().cpu().numpy().reshape(shape), want_d) <= 1e-3
