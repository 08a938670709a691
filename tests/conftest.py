"""Shared test set-up: import paths, markers, native builds, helpers.

Tests marked ``gpu`` need a CUDA device; everything else runs on CPU.
The checker (oracle/) is imported only from tests.
"""
import glob
import importlib.machinery
import importlib.util
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "dosecuda-jax_b200")
for p in (PKG_DIR, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    lib = os.path.join(PKG_DIR, "dosecuda_b200", "libpb_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(PKG_DIR, "csrc")], check=True)
    for name in ("liboracle.so", "libport32.so"):
        if not os.path.exists(os.path.join(ROOT, "oracle", name)):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), name], check=True)


_ensure_built()


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def load_reference_module():
    """The reference's own dose_kernels built from its sources (oracle/_ref),
    or None when it has not been built."""
    paths = glob.glob(os.path.join(ROOT, "oracle", "_ref", "dose_kernels*.so"))
    if not paths:
        return None
    if "dose_kernels" in sys.modules and getattr(sys.modules["dose_kernels"], "__file__", "") == paths[0]:
        return sys.modules["dose_kernels"]
    loader = importlib.machinery.ExtensionFileLoader("dose_kernels", paths[0])
    spec = importlib.util.spec_from_file_location("dose_kernels", paths[0], loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def max_rel(a, b, ref_max=None):
    """max |a - b| / max(ref)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = float(np.abs(b).max()) if ref_max is None else float(ref_max)
    return float(np.abs(a - b).max() / m) if m > 0 else float(np.abs(a - b).max())


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle.  With a CUDA device present its smoothing takes the
    six directions from the device's sincosf (pb_smooth_dirs), as the
    reference and the kernels do; without one, the C library's."""
    from oracle import oracle as O
    O.load()
    if cuda_available():
        from dosecuda_b200 import _lib
        O.set_smooth_dirs(*_lib.smooth_dirs())
    return O


@pytest.fixture(scope="session")
def reference_module():
    mod = load_reference_module()
    if mod is None:
        pytest.skip("the reference module oracle/_ref/dose_kernels*.so is not built")
    return mod
