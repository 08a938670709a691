"""The reference-compatible plan API on the host: beam-model parsing, spot
bookkeeping, phantoms, NRRD I/O, the dose_kernels attribute contract and
the errors raised before any device work."""
import glob
import os
import types

import numpy as np
import pytest

from conftest import PKG_DIR


@pytest.fixture(scope="module")
def plan():
    from dosecuda_b200.plan_impt import IMPTPlan
    return IMPTPlan()


LUT_DIR = os.path.join(PKG_DIR, "dosecuda_b200", "lookuptables", "protons", "HitachiProbeatJHU")


def test_machine_models_parse(plan):
    assert list(plan.dicom_rangeshifter_label.astype(str)) == ["0", "4"]
    for model, folder in zip(plan.beam_models, ["RS0", "RS4"]):
        assert model.VSADX == 1340.0 and model.VSADY == 1930.0
        assert model.divergence_params.shape == (98, 5)
        assert model.lut_depths.shape == (98, 400) and model.lut_depths.dtype == np.float32
        files = sorted(glob.glob(os.path.join(LUT_DIR, folder, "energy_*.csv")))
        assert len(files) == 98
        for e, f in enumerate(files):
            rows = np.loadtxt(f, delimiter=",", skiprows=4, max_rows=400, dtype=np.float64)
            head = np.loadtxt(f, delimiter=",", skiprows=1, max_rows=1, dtype=np.float64)
            assert np.array_equal(model.lut_depths[e], rows[:, 0].astype(np.float32))
            assert np.array_equal(model.lut_sigmas[e], rows[:, 1].astype(np.float32))
            assert np.array_equal(model.lut_idds[e], rows[:, 2].astype(np.float32))
            assert np.array_equal(model.divergence_params[e], head.astype(np.float32))
    m = plan.beam_models[0]
    assert m.energyIDFromLabel(70.2) == 0 and m.energyIDFromLabel(228.7) == 97
    with pytest.raises(Exception, match="Energy ID not found"):
        m.energyIDFromLabel(1.0)


def test_beam_spot_api():
    from dosecuda_b200.plan_impt import IMPTBeam
    b = IMPTBeam()
    b.addSingleSpot(1.0, 2.0, 0.5, 3)
    assert b.spot_list.shape == (4,) and b.n_spots == 1      # the reference's 1-D quirk
    b.addSingleSpot(-1.0, 0.0, 1.5, 4)
    assert b.spot_list.shape == (2, 4) and b.spot_list.dtype == np.float32
    cp = types.SimpleNamespace(ScanSpotPositionMap=[0, 0, 5, 5, -5, 5],
                               ScanSpotMetersetWeights=[0.1, 0.2, 0.3])
    b.addSpotData(cp, 7)
    assert b.n_spots == 5 and list(b.spot_list[-1]) == [-5.0, 5.0, 0.3, 7.0]
    b.changeSpotEnergy(2)
    assert set(b.spot_list[:, 3]) == {2.0}
    c = IMPTBeam(b)
    assert c.n_spots == 5 and c.spot_list is b.spot_list
    b.resetSpots()
    assert b.spot_list.shape == (0, 4) and b.n_spots == 0


def test_plan_add_beam_names(plan):
    from dosecuda_b200.plan_impt import IMPTBeam, IMPTPlan
    p = IMPTPlan()
    p.addBeam(IMPTBeam())
    p.addBeam(IMPTBeam())
    assert [b.BeamName for b in p.beam_list] == ["PBS_Beam1", "PBS_Beam2"]
    p.addPrescription(60.0, "PTV", 0.02)
    assert p.Prescriptions[0].ROIName == "PTV"


def test_cube_phantom_like_reference():
    from dosecuda_b200.plan_impt import IMPTDoseGrid
    g = IMPTDoseGrid()
    g.createCubePhantom()
    assert g.HU.shape == (138, 138, 138) and g.HU.dtype == np.float32
    assert np.allclose(g.origin, -207.0) and np.allclose(g.spacing, 3.0)
    edge = round(10.0 / 3.0)
    assert g.HU[0, 0, 0] == -1000.0 and g.HU[edge, edge, edge] == 0.0
    assert g.HU[edge - 1, 70, 70] == -1000.0


def test_couch_model():
    from dosecuda_b200.plan_impt import IMPTDoseGrid
    g = IMPTDoseGrid()
    g.createCubePhantom(size=[20, 30, 20], spacing=5.0)
    g.applyCouchModel(couch_wet=8.0)
    n = int(50.0 / 5.0)
    assert np.allclose(g.HU[:, -n:, :], ((8.0 / (n * 5.0)) - 1.0) * 1000.0)


def test_nrrd_roundtrip(tmp_path):
    from dosecuda_b200 import nrrd
    from dosecuda_b200.plan_impt import IMPTDoseGrid
    rng = np.random.default_rng(0)
    vol = rng.normal(size=(5, 6, 7)).astype(np.float32)
    for compress in (False, True):
        p = str(tmp_path / f"v{compress}.nrrd")
        nrrd.write(p, vol, [-1.0, 2.0, 3.5], [2.0, 2.0, 2.5], compress=compress)
        v2, o, s = nrrd.read(p)
        assert np.array_equal(v2, vol) and np.allclose(o, [-1, 2, 3.5]) and np.allclose(s, [2, 2, 2.5])
    g = IMPTDoseGrid()
    g.createCubePhantom(size=[8, 9, 10], spacing=4.0)
    g.dose = np.ones(g.HU.shape, np.float32)
    g.beam_doses = [g.dose * 2]
    g.writeDoseNRRD(str(tmp_path / "d.nrrd"), individual_beams=True, dose_type="PHYSICAL")
    v, _, _ = nrrd.read(str(tmp_path / "d_beam01.nrrd"))
    assert np.allclose(v, 2.0)
    g.writeDoseNRRD(str(tmp_path / "e.nrrd"))
    v, _, _ = nrrd.read(str(tmp_path / "e.nrrd"))
    assert np.allclose(v, 1.1)
    g.writeCTNRRD(str(tmp_path / "ct.nrrd"))
    g2 = IMPTDoseGrid()
    g2.loadCTNRRD(str(tmp_path / "ct.nrrd"))
    assert np.array_equal(g2.HU, g.HU) and np.allclose(g2.origin, g.origin)
    with pytest.raises(Exception, match="extension"):
        g.writeDoseNRRD(str(tmp_path / "d.txt"))
    with pytest.raises(Exception, match="Unknown dose type"):
        g.writeDoseNRRD(str(tmp_path / "d.nrrd"), dose_type="X")


class _Obj:
    pass


def _args():
    from dosecuda_b200.plan_impt import IMPTPlan
    model = IMPTPlan().beam_models[0]
    vol = _Obj()
    vol.voxel_data = np.zeros((4, 4, 4), np.float32)
    vol.spacing = np.ones(3, np.float32)
    vol.origin = np.zeros(3, np.float32)
    beam = _Obj()
    beam.iso = np.zeros(3, np.float32)
    beam.gantry_angle = 0.0
    beam.couch_angle = 0.0
    beam.spot_list = np.zeros((2, 4), np.float32)
    return model, vol, beam


def test_dose_kernels_attribute_contract():
    """dosemodule.cu:23-101: rank/dtype -> ValueError with the reference's
    message, missing attribute -> AttributeError, non-number -> TypeError;
    all raised before any device work."""
    from dosecuda_b200 import dose_kernels as dk
    model, vol, beam = _args()
    vol.voxel_data = np.zeros((4, 4, 4), np.float64)
    with pytest.raises(ValueError, match="'voxel_data' must be 3-dimensional and of type float."):
        dk.proton_raytrace_cuda(model, vol, beam, 0)
    model, vol, beam = _args()
    beam.spot_list = np.zeros(4, np.float32)          # 1-spot beams are 1-D: rejected
    with pytest.raises(ValueError, match="'spot_list' must be 2-dimensional"):
        dk.proton_spot_cuda(model, vol, vol, beam, 0)
    model, vol, beam = _args()
    del beam.iso
    with pytest.raises(AttributeError):
        dk.proton_raytrace_cuda(model, vol, beam, 0)
    model, vol, beam = _args()
    beam.gantry_angle = "90"
    with pytest.raises(TypeError):
        dk.proton_raytrace_cuda(model, vol, beam, 0)


def test_plan_errors_before_device_work(plan):
    from dosecuda_b200.plan_impt import IMPTBeam, IMPTDoseGrid
    g = IMPTDoseGrid()
    g.createCubePhantom(size=[8, 8, 8], spacing=3.0)
    g.spacing = np.array([3.0, 3.0, 2.0])
    with pytest.raises(Exception, match="isotropic"):
        g.computeIMPTPlan(plan)
    g.spacing = np.array([3.0, 3.0, 3.0])
    b = IMPTBeam()
    b.dicom_rangeshifter_label = "9"
    b.addSingleSpot(0, 0, 1, 10)
    from dosecuda_b200.plan_impt import IMPTPlan
    p = IMPTPlan()
    p.addBeam(b)
    with pytest.raises(SystemExit):
        g._specs(p, p.beam_list)


def test_phantoms_are_seeded():
    from dosecuda_b200 import phantoms
    a = phantoms.small_heterogeneous(seed=4)
    b = phantoms.small_heterogeneous(seed=4)
    assert np.array_equal(a.grid.HU, b.grid.HU)
    assert all(np.array_equal(x.spot_list, y.spot_list)
               for x, y in zip(a.plan.beam_list, b.plan.beam_list))
    c = phantoms.water_cube()
    assert c.grid.HU.shape == (120, 120, 120) and c.n_spots == 121 * 10
    assert (c.grid.HU == 0).sum() == 80 ** 3


def _ion_plan_dataset(labels):
    """A synthetic RT Ion Plan in the shape pydicom gives (attributes and
    sequences): two beams, the second with range shifter '4'; control points
    in pairs (layer start with spots, layer end), as planning systems write
    them."""
    ns = types.SimpleNamespace

    def layer(energy, xy, mu, first=None):
        cp = ns(NominalBeamEnergy=float(energy), ScanSpotPositionMap=list(np.ravel(xy)),
                ScanSpotMetersetWeights=list(mu))
        if first is not None:
            cp.GantryAngle, cp.PatientSupportAngle, cp.IsocenterPosition = first
        end = ns(NominalBeamEnergy=float(energy), ScanSpotPositionMap=list(np.ravel(xy)),
                 ScanSpotMetersetWeights=[0.0] * len(mu))
        return [cp, end]

    b1 = ns(BeamName="RAO", NumberOfRangeShifters=0,
            IonControlPointSequence=layer(labels[40], [[0, 0], [5, 0]], [1.0, 2.0],
                                          (30.0, 0.0, [1.0, 2.0, 3.0]))
            + layer(labels[45], [[0, 5]], [0.5]))
    b2 = ns(BeamName="LAO", BeamDescription="second", NumberOfRangeShifters=1,
            RangeShifterSequence=[ns(RangeShifterID="4")],
            IonControlPointSequence=layer(labels[20], [[-5, -5], [5, 5], [0, 0]],
                                          [1.0, 1.0, 3.0], (330.0, 90.0, [4.0, 5.0, 6.0])))
    return ns(IonBeamSequence=[b1, b2],
              FractionGroupSequence=[ns(NumberOfFractionsPlanned="30")])


def test_read_plan_dicom_from_dataset(plan):
    """readPlanDicom (plan_impt.py:635-674) on a dataset already read: beams,
    angles, isocentres, range shifters, spots of the even control points with
    their energy ids, and the fraction count."""
    from dosecuda_b200.plan_impt import IMPTPlan
    p = IMPTPlan()
    labels = p.beam_models[0].energy_labels
    p.readPlanDicom(_ion_plan_dataset(labels))
    assert p.n_fractions == 30.0 and p.n_beams == 2
    b1, b2 = p.beam_list
    assert (b1.gantry_angle, b1.couch_angle) == (30.0, 0.0)
    assert (b2.gantry_angle, b2.couch_angle) == (330.0, 90.0)
    assert b1.iso.dtype == np.float32 and list(b1.iso) == [1.0, 2.0, 3.0]
    assert b1.dicom_rangeshifter_label == "0" and b2.dicom_rangeshifter_label == "4"
    assert b1.BeamName == "RAO" and b2.BeamDescription == "second"
    assert b1.BeamDescription == "PBS_Beam 1"
    assert b1.spot_list.dtype == np.float32 and b1.spot_list.shape == (3, 4)
    assert np.array_equal(b1.spot_list, np.array([[0, 0, 1, 40], [5, 0, 2, 40], [0, 5, 0.5, 45]],
                                                 np.float32))
    assert b1.n_spots == 3 and b2.n_spots == 3
    assert np.array_equal(b2.spot_list[:, 3], [20, 20, 20])


def test_read_plan_dicom_file_needs_pydicom(plan, tmp_path):
    import importlib.util
    if importlib.util.find_spec("pydicom") is not None:
        pytest.skip("pydicom is installed")
    with pytest.raises(ImportError, match="pydicom"):
        plan.readPlanDicom(str(tmp_path / "plan.dcm"))


class _FakeItem:
    pass


class _FakeRTDose:
    """Stands in for a pydicom RT Dose dataset: the attributes writeDoseDCM
    edits, and save_as recording what would be written."""

    saved = []

    def __init__(self):
        self.SeriesDescription = "TPS dose"
        self.DoseSummationType = "PLAN"
        self.DoseType = "PHYSICAL"
        self.DoseGridScaling = 1.0
        self.PixelData = b""
        item = _FakeItem()
        item.ReferencedSOPInstanceUID = "1.2.3"
        self.ReferencedRTPlanSequence = [item]

    def save_as(self, path):
        _FakeRTDose.saved.append((path, dict(self.__dict__)))


def test_write_dose_dcm_edits_a_reference_dataset(tmp_path):
    """writeDoseDCM (plan.py:133-171) on a dataset object: the plan dose and
    per-beam doses as uint16 of dose * 500 * RBE with DoseGridScaling 0.002,
    a new referenced plan UID per file, the reference dataset untouched."""
    from dosecuda_b200.plan import DoseGrid
    g = DoseGrid()
    rng = np.random.default_rng(0)
    g.dose = rng.uniform(0.0, 60.0, (3, 4, 5)).astype(np.float32)
    g.beam_doses = [g.dose * 0.25, g.dose * 0.75]
    ref = _FakeRTDose()
    _FakeRTDose.saved.clear()
    with pytest.raises(Exception, match="dcm extension"):
        g.writeDoseDCM(str(tmp_path / "d.nrrd"), ref)
    with pytest.raises(Exception, match="Unknown dose type"):
        g.writeDoseDCM(str(tmp_path / "d.dcm"), ref, dose_type="RBE")
    g.writeDoseDCM(str(tmp_path / "d.dcm"), ref)
    g.writeDoseDCM(str(tmp_path / "d.dcm"), ref, dose_type="PHYSICAL", individual_beams=True)
    paths = [p for p, _ in _FakeRTDose.saved]
    assert paths == [str(tmp_path / n) for n in ("d.dcm", "d_beam01.dcm", "d_beam02.dcm")]
    plan_ds, b1, b2 = (d for _, d in _FakeRTDose.saved)
    assert plan_ds["SeriesDescription"] == "TPS dose_DoseCUDA"
    assert plan_ds["DoseSummationType"] == "PLAN" and plan_ds["DoseType"] == "EFFECTIVE"
    assert b1["DoseSummationType"] == "BEAM" and b1["DoseType"] == "PHYSICAL"
    assert plan_ds["DoseGridScaling"] == 0.002
    px = np.frombuffer(plan_ds["PixelData"], "<u2").reshape(g.dose.shape)
    assert np.array_equal(px, np.array(g.dose * 500.0 * 1.1, dtype=np.uint16))
    px2 = np.frombuffer(b2["PixelData"], "<u2").reshape(g.dose.shape)
    assert np.array_equal(px2, np.array(g.beam_doses[1] * 500.0 * 1.0, dtype=np.uint16))
    uids = {d["ReferencedRTPlanSequence"][0].ReferencedSOPInstanceUID for d in (plan_ds, b1, b2)}
    import re
    # valid DICOM UIDs: dotted numbers, at most 64 characters
    assert len(uids) == 3 and all(re.fullmatch(r"[0-9]+(\.[0-9]+)+", u) and len(u) <= 64
                                  for u in uids)
    # the reference dataset itself is not modified
    assert ref.SeriesDescription == "TPS dose" and ref.PixelData == b""
    assert ref.ReferencedRTPlanSequence[0].ReferencedSOPInstanceUID == "1.2.3"


def test_write_dose_dcm_from_a_file_needs_pydicom(tmp_path):
    from dosecuda_b200.plan import DoseGrid
    try:
        import pydicom  # noqa: F401
        pytest.skip("pydicom is installed")
    except ImportError:
        pass
    g = DoseGrid()
    g.dose = np.zeros((2, 2, 2), np.float32)
    with pytest.raises(ImportError, match="pydicom"):
        g.writeDoseDCM(str(tmp_path / "d.dcm"), str(tmp_path / "ref.dcm"))


def test_write_ct_nifti_roundtrip(tmp_path):
    """writeCTNIFTI (plan.py:214-224): NIfTI-1, gzip, LPS stored as RAS as an
    ITK writer stores it; read back equal."""
    import gzip
    import struct

    from dosecuda_b200 import nifti
    from dosecuda_b200.plan import DoseGrid
    g = DoseGrid()
    g.HU = np.random.default_rng(1).uniform(-1000, 2000, (4, 5, 6)).astype(np.float32)
    g.origin = np.array([-10.0, 20.0, -30.5])
    g.spacing = np.array([1.5, 1.5, 2.0])
    with pytest.raises(Exception, match="nii.gz"):
        g.writeCTNIFTI(str(tmp_path / "ct.nii"))
    path = str(tmp_path / "ct.nii.gz")
    g.writeCTNIFTI(path)
    vol, origin, spacing = nifti.read(path)
    assert np.array_equal(vol, g.HU)
    assert np.allclose(origin, g.origin) and np.allclose(spacing, g.spacing)
    raw = gzip.decompress(open(path, "rb").read())
    assert struct.unpack_from("<8h", raw, 40)[:4] == (3, 6, 5, 4)
    assert struct.unpack_from("<hh", raw, 70) == (16, 32)
    assert struct.unpack_from("<4f", raw, 280) == (-1.5, 0.0, 0.0, 10.0)
    assert struct.unpack_from("<3f", raw, 256) == (0.0, 0.0, 1.0)
