"""Drop-in module name ``dose_kernels`` (the reference's CPython extension,
DoseCUDA/dose_kernels/dosemodule.cu:560-595) for the proton entry points."""
import os as _os
import sys as _sys

_pkg_root = _os.path.dirname(_os.path.dirname(_os.path.abspath(__file__)))
if _pkg_root not in _sys.path:
    _sys.path.insert(0, _pkg_root)

from dosecuda_b200.dose_kernels import proton_raytrace_cuda, proton_spot_cuda  # noqa: E402,F401
