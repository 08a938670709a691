"""B200-native proton pencil-beam dose (DoseCUDA IMPT path) on sm_100a.

Public API mirrors DoseCUDA's IMPT classes (DoseCUDA/__init__.py:1):
    IMPTDoseGrid, IMPTPlan, IMPTBeam
plus the device-resident engine (``engine.DevicePlan``), the
differentiable dose (``autograd.dose``) and the ``dose_kernels`` drop-in.
"""
from ._lib import PbError  # noqa: F401  (loads libpb_b200.so; fails loudly if missing)
from .plan_impt import IMPTBeam, IMPTBeamModel, IMPTDoseGrid, IMPTPlan  # noqa: F401
from .plan import Beam, DoseGrid, Plan, Prescription, VolumeObject  # noqa: F401

__all__ = ["IMPTDoseGrid", "IMPTPlan", "IMPTBeam", "IMPTBeamModel"]
