"""Generate the golden fixtures of this directory from the reference itself.

Runs the reference's own CUDA module (dose_kernels, built from the reference
sources into oracle/_ref by `make -C oracle ref`) on a CUDA device, through
its public entry points proton_raytrace_cuda / proton_spot_cuda
(DoseCUDA/dose_kernels/dosemodule.cu:560-580), for small seeded cases, and
stores inputs and outputs as compressed .npz files:

    python tests/golden/make_golden.py [out_dir]

Each file holds the CT (HU), grid (origin, spacing), the machine's HU->RLSP
curve, per beam the gantry/couch angles, isocentre, range-shifter label and
spot list, and the reference's smoothed WET and dose for each beam.  The CPU
tests check the oracle against these files; nothing here is used by the
product.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "dosecuda-jax_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)

from conftest import load_reference_module  # noqa: E402
from dosecuda_b200 import phantoms  # noqa: E402
from dosecuda_b200.plan import VolumeObject  # noqa: E402
from dosecuda_b200.plan_impt import IMPTBeam, IMPTDoseGrid, _hu_curve  # noqa: E402


def cube_case():
    """Cube phantom (plan.py:226-232) at 5 mm with a ring of 8 spots of
    increasing energy id, the reference's own comparison plan shape
    (tests/compare_cuda_jax.py:32-39) scaled to the smaller grid."""
    g = IMPTDoseGrid()
    g.createCubePhantom(size=[30, 30, 30], spacing=5.0)
    plan = phantoms._new_plan()
    beam = IMPTBeam()
    beam.dicom_rangeshifter_label = '0'
    for e in range(8):
        th = 2.0 * 3.14159 * e / 8
        beam.addSingleSpot(30.0 * np.cos(th), 30.0 * np.sin(th), 0.2, e * 3)
    plan.addBeam(beam)
    return "cube_ring", g, plan


def hetero_case():
    c = phantoms.heterogeneous(seed=5, angles=(0.0, 135.0), n_spots=240, shape=(24, 28, 32),
                               spacing=4.0, n_slabs=1, n_spheres=2, semi_range=(10.0, 16.0),
                               centre_jitter=5.0, body_inset=12.0)
    return "hetero_two_beams", c.grid, c.plan


def couch_rs4_case():
    """Couch rotation, off-axis gantry and the range-shifter model RS4
    (whose lowest energies have R80 < 0.2 mm, the halo clamp edge)."""
    c = phantoms.heterogeneous(seed=9, angles=(45.0,), n_spots=150, shape=(26, 24, 30),
                               spacing=4.0, n_slabs=1, n_spheres=1, semi_range=(10.0, 14.0),
                               centre_jitter=4.0, body_inset=12.0)
    b = c.plan.beam_list[0]
    b.couch_angle = 90.0
    b.dicom_rangeshifter_label = '4'
    sl = np.array(b.spot_list, dtype=np.single)
    sl[: min(12, len(sl)), 3] = np.arange(min(12, len(sl)))  # low RS4 energies too
    b.spot_list = sl
    return "couch90_rs4", c.grid, c.plan


def run(out_dir):
    ref = load_reference_module()
    if ref is None:
        raise SystemExit("oracle/_ref/dose_kernels is not built (make -C oracle ref)")
    os.makedirs(out_dir, exist_ok=True)
    curve = _hu_curve("HitachiProbeatJHU")
    for name, g, plan in (cube_case(), hetero_case(), couch_rs4_case()):
        rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
        vol = VolumeObject()
        vol.voxel_data = rlsp
        vol.origin = np.array(g.origin, dtype=np.single)
        vol.spacing = np.array(g.spacing, dtype=np.single)
        rec = {"hu": np.asarray(g.HU, np.float32), "origin": np.asarray(g.origin, np.float64),
               "spacing": np.asarray(g.spacing, np.float64), "curve_hu": curve[0],
               "curve_rlsp": curve[1], "n_beams": np.int64(len(plan.beam_list))}
        labels = list(plan.dicom_rangeshifter_label.astype(str))
        for b, beam in enumerate(plan.beam_list):
            model = plan.beam_models[labels.index(beam.dicom_rangeshifter_label)]
            wet = ref.proton_raytrace_cuda(model, vol, beam, 0)
            wv = VolumeObject()
            wv.voxel_data = np.array(wet, dtype=np.single)
            wv.origin = vol.origin
            wv.spacing = vol.spacing
            beam.spot_list = np.array(beam.spot_list, dtype=np.single).reshape(-1, 4)
            dose = ref.proton_spot_cuda(model, vol, wv, beam, 0)
            rec[f"b{b}_gantry"] = np.float64(beam.gantry_angle)
            rec[f"b{b}_couch"] = np.float64(beam.couch_angle)
            rec[f"b{b}_iso"] = np.asarray(beam.iso, np.float32)
            rec[f"b{b}_label"] = np.array(beam.dicom_rangeshifter_label)
            rec[f"b{b}_spots"] = beam.spot_list
            rec[f"b{b}_wet"] = np.asarray(wet, np.float32)
            rec[f"b{b}_dose"] = np.asarray(dose, np.float32)
        path = os.path.join(out_dir, f"{name}.npz")
        np.savez_compressed(path, **rec)
        print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    run(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
