"""Drop-in package name: ``from DoseCUDA import IMPTDoseGrid, IMPTPlan, IMPTBeam``
(DoseCUDA/__init__.py:1) resolves to the B200 implementation when
``dosecuda-jax_b200/compat`` and ``dosecuda-jax_b200`` are on sys.path.
The photon (IMRT) classes of the reference are not provided."""
import os as _os
import sys as _sys

_pkg_root = _os.path.dirname(_os.path.dirname(_os.path.dirname(_os.path.abspath(__file__))))
if _pkg_root not in _sys.path:
    _sys.path.insert(0, _pkg_root)

from dosecuda_b200.plan_impt import IMPTBeam, IMPTDoseGrid, IMPTPlan  # noqa: E402,F401

__all__ = ['IMPTDoseGrid', 'IMPTPlan', 'IMPTBeam']
