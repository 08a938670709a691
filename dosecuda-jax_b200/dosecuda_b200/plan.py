"""Plan, beam and dose-grid containers (mirror of DoseCUDA/plan.py).

Same classes, attribute names and defaults as the reference so that code
written against ``DoseCUDA.plan`` runs unchanged:
  VolumeObject (plan.py:6-11), Prescription (:14-19), DoseGrid (:22-232),
  Beam (:235-243), Plan (:246-268).
NRRD and NIfTI volume I/O is served by the package's own readers/writers.
The RT Dose writer (writeDoseDCM) edits a reference RT Dose dataset: one
read through pydicom from a path, or any dataset object already read (the
same attributes and save_as).  DICOM CT reading and SimpleITK resampling
need pydicom/SimpleITK and raise NotImplementedError with that reason.
"""
from __future__ import annotations

import copy
import uuid

import numpy as np

from . import nifti, nrrd


def generate_uid() -> str:
    """A new DICOM UID: pydicom's generator when pydicom is installed, else
    the UUID-derived form 2.25.<128-bit integer> of DICOM PS3.5 B.2."""
    try:
        from pydicom.uid import generate_uid as gen
        return str(gen())
    except ImportError:
        return "2.25.%d" % uuid.uuid4().int


def _dataset(ref):
    """A dataset to edit: read from a path with pydicom (force=True, as the
    reference does), or a deep copy of a dataset object already read."""
    if isinstance(ref, (str, bytes)) or hasattr(ref, "__fspath__"):
        try:
            import pydicom
        except ImportError as e:
            raise ImportError("reading a DICOM file needs pydicom; pass a dataset already "
                              "read instead") from e
        return pydicom.dcmread(ref, force=True)
    return copy.deepcopy(ref)


class VolumeObject:

    def __init__(self):
        self.origin = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.spacing = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.voxel_data = []


class Prescription:

    def __init__(self):
        self.TargetPrescriptionDose = 0.0
        self.ROIName = None
        self.TargetUnderdoseVolumeFraction = 0.0


def _rbe(dose_type: str) -> float:
    if dose_type == "EFFECTIVE":
        return 1.1
    if dose_type == "PHYSICAL":
        return 1.0
    raise Exception("Unknown dose type: %s" % dose_type)


class DoseGrid:

    def __init__(self):
        self.origin = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.spacing = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.size = np.array([0, 0, 0])
        self.HU = []
        self.dose = []
        self.beam_doses = []
        self.FrameOfReferenceUID = ""

    # -- CT input ---------------------------------------------------------
    def loadCTNRRD(self, ct_path):
        """Load a CT volume (HU) from NRRD (plan.py:33-41)."""
        vol, origin, spacing = nrrd.read(ct_path)
        self.origin = np.array(origin)
        self.spacing = np.array(spacing)
        self.HU = np.array(vol, dtype=np.single)
        self.size = np.array(self.HU.shape)

    def loadCTDCM(self, ct_path):
        raise NotImplementedError("loadCTDCM reads DICOM series through SimpleITK, "
                                  "which this package does not depend on")

    def resampleCT(self, new_spacing, new_size, new_origin):
        raise NotImplementedError("resampleCT uses SimpleITK's resampler")

    def resampleCTfromSpacing(self, spacing):
        raise NotImplementedError("resampleCTfromSpacing uses SimpleITK's resampler")

    def resampleCTfromReferenceDose(self, ref_dose_path):
        raise NotImplementedError("resampleCTfromReferenceDose reads DICOM through pydicom")

    def applyCouchModel(self, couch_wet=8.0):
        """Replace the last 50 mm of rows with a couch of the given WET
        (plan.py:126-131)."""
        spacing = self.spacing[0]
        n_voxels = int(50.0 / spacing)
        hu_override_value = ((couch_wet / (n_voxels * spacing)) - 1.0) * 1000.0
        self.HU[:, -n_voxels:, :] = hu_override_value

    # -- output -------------------------------------------------------------
    def writeDoseDCM(self, dose_path, ref_dose_path, dose_type="EFFECTIVE",
                     individual_beams=False):
        """The plan dose (or each beam's) as RT Dose files built on a
        reference RT Dose (plan.py:133-171): its SeriesDescription + "_DoseCUDA",
        DoseSummationType PLAN (BEAM per beam), DoseType, a new referenced
        plan UID, pixel data dose * 500 * RBE as uint16 with DoseGridScaling
        0.002.  ref_dose_path is a file (read with pydicom) or a dataset
        already read, copied for every output file.  The pixel data is
        stored as the array's little-endian bytes."""
        if not dose_path.endswith(".dcm"):
            raise Exception("Dose path must have .dcm extension")
        rbe = _rbe(dose_type)
        if individual_beams:
            outs = [(dose_path.replace(".dcm", "_beam%02i.dcm" % (i + 1)), d, "BEAM")
                    for i, d in enumerate(self.beam_doses)]
        else:
            outs = [(dose_path, self.dose, "PLAN")]
        for path, dose, summation in outs:
            ref_dose = _dataset(ref_dose_path)
            ref_dose.SeriesDescription = ref_dose.SeriesDescription + "_DoseCUDA"
            ref_dose.DoseSummationType = summation
            ref_dose.DoseType = dose_type
            ref_dose.ReferencedRTPlanSequence[0].ReferencedSOPInstanceUID = generate_uid()
            dose_dcm = np.array(np.asarray(dose) * 500.0 * rbe, dtype=np.uint16)
            ref_dose.PixelData = dose_dcm.astype("<u2").tobytes()
            ref_dose.DoseGridScaling = 0.002
            ref_dose.save_as(path)

    def writeDoseNRRD(self, dose_path, individual_beams=False, dose_type="EFFECTIVE"):
        """Write the plan dose (or each beam's) times RBE (plan.py:173-199)."""
        if not dose_path.endswith(".nrrd"):
            raise Exception("Dose path must have .nrrd extension")
        rbe = _rbe(dose_type)
        if individual_beams:
            for i, beam_dose in enumerate(self.beam_doses):
                nrrd.write(dose_path.replace(".nrrd", "_beam%02i.nrrd" % (i + 1)),
                           np.array(beam_dose * rbe, dtype=np.single), self.origin,
                           self.spacing)
        else:
            nrrd.write(dose_path, np.array(self.dose * rbe, dtype=np.single), self.origin,
                       self.spacing)

    def writeCTNRRD(self, ct_path):
        if not ct_path.endswith(".nrrd"):
            raise Exception("CT path must have .nrrd extension")
        nrrd.write(ct_path, np.asarray(self.HU), self.origin, self.spacing)

    def writeCTNIFTI(self, ct_path):
        """The CT (HU) as gzip-compressed NIfTI-1 (plan.py:214-224)."""
        if not ct_path.endswith(".nii.gz"):
            raise Exception("CT path must have .nii.gz extension")
        nifti.write(ct_path, np.asarray(self.HU), self.origin, self.spacing)

    # -- phantoms -----------------------------------------------------------
    def createCubePhantom(self, size=[138, 138, 138], spacing=3.0):
        """Water cube with a 10 mm air rim, centred on the origin
        (plan.py:226-232)."""
        self.origin = np.array([-size[0] * spacing / 2.0, -size[1] * spacing / 2.0,
                                -size[2] * spacing / 2.0])
        self.spacing = np.array([spacing, spacing, spacing])
        self.size = np.array(size)
        edge = round(10.0 / spacing)
        self.HU = np.ones(size, dtype=np.single) * -1000.0
        self.HU[edge:-edge, edge:-edge, edge:-edge] = 0.0


class Beam:

    def __init__(self):
        self.iso = np.array([0.0, 0.0, 0.0], dtype=np.single)
        self.gantry_angle = 0.0
        self.collimator_angle = 0.0
        self.couch_angle = 0.0
        self.BeamName = None
        self.BeamDescription = None


class Plan:

    def __init__(self):
        self.n_beams = 0
        self.n_fractions = 1
        self.beam_list = []
        self.RTPlanLabel = None
        self.Prescriptions = []

    def addPrescription(self, TargetPrescriptionDose, ROIName, TargetUnderdoseVolumeFraction):
        rx = Prescription()
        rx.TargetPrescriptionDose = TargetPrescriptionDose
        rx.ROIName = ROIName
        rx.TargetUnderdoseVolumeFraction = TargetUnderdoseVolumeFraction
        self.Prescriptions.append(rx)

    def addBeam(self, beam):
        if not beam.BeamName:
            beam.BeamName = f'PBS_Beam{self.n_beams + 1}'
        if not beam.BeamDescription:
            beam.BeamDescription = f'PBS_Beam {self.n_beams + 1}'
        self.beam_list.append(beam)
        self.n_beams += 1
