"""B200-native proton pencil-beam dose (DoseCUDA IMPT path) on sm_100a.

Public API mirrors DoseCUDA's IMPT classes (DoseCUDA/__init__.py:1):
    IMPTDoseGrid, IMPTPlan, IMPTBeam
plus the device-resident engine (``engine.DevicePlan``), the
differentiable dose (``autograd.dose``) and the ``dose_kernels`` drop-in.

Importing the package builds no device state and does not load
libpb_b200.so: the plan classes, beam models and synthetic phantoms are
host-side data.  The library is loaded by the first computation (through
``engine`` / ``_lib``), which raises ImportError when it is missing -- the
dose path has no CPU fallback.
"""
from .plan_impt import IMPTBeam, IMPTBeamModel, IMPTDoseGrid, IMPTPlan  # noqa: F401
from .plan import Beam, DoseGrid, Plan, Prescription, VolumeObject  # noqa: F401

__all__ = ["IMPTDoseGrid", "IMPTPlan", "IMPTBeam", "IMPTBeamModel", "PbError"]


def __getattr__(name):
    if name == "PbError":
        from ._lib import PbError
        return PbError
    raise AttributeError(f"module 'dosecuda_b200' has no attribute {name!r}")
