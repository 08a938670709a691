"""IMPT plan API (mirror of DoseCUDA/plan_impt.py) on the B200 kernels.

Class names, attributes, method names, arguments and error behaviour follow
the reference (plan_impt.py:63-342); the dose computation goes through the
package's CUDA kernels with all beams of a plan in one launch and the CT,
RLSP, WET and dose kept on the device.

Beyond the reference:
  IMPTDoseGrid.prepareIMPTPlan      device-resident plan for repeated use
  IMPTDoseGrid.computeIMPTPlanGradient
                                    objective + spot-weight gradient
"""
from __future__ import annotations

import ctypes
import os
import sys
import weakref

import numpy as np
import pandas as pd
import torch

from . import nrrd
from .plan import Beam, DoseGrid, Plan, Prescription, VolumeObject  # noqa: F401

_PKG = os.path.dirname(os.path.abspath(__file__))


def _engine():
    """The device engine.  Imported on first use, so that the plan classes,
    beam models and lookup tables can be built without loading
    libpb_b200.so; every dose computation goes through here and raises
    ImportError when the library is missing (there is no CPU path)."""
    from . import engine
    return engine


def resource_filename(rel_path: str) -> str:
    """Path of a package data file (the reference uses pkg_resources)."""
    return os.path.join(_PKG, rel_path)


class IMPTBeamModel():
    """Lookup-table beam model of one range-shifter setting
    (plan_impt.py:63-149): VSADX/VSADY from machine_geometry.csv; per energy
    divergence_params (energy, R80, A, B, C) and the first 400 rows of
    depth / sigma / IDD from energy_NNN.csv."""

    def __init__(self, dicom_rangeshifter_label, path_to_model, folder_rangeshifter_label):

        self.dicom_rangeshifter_label = dicom_rangeshifter_label

        machine_geometry_path = resource_filename(os.path.join(path_to_model, "machine_geometry.csv"))

        self.VSADX = None
        self.VSADY = None

        for line in open(machine_geometry_path, "r"):
            if line.startswith("VSADX"):
                self.VSADX = float(line.split(',')[1])
            if line.startswith("VSADY"):
                self.VSADY = float(line.split(',')[1])

        if self.VSADX is None:
            raise Exception("VSADX not found in machine_geometry.csv")
        if self.VSADY is None:
            raise Exception("VSADY not found in machine_geometry.csv")

        energy_list_path = resource_filename(os.path.join(path_to_model, folder_rangeshifter_label,
                                                          "energies.csv"))
        self.energy_table = pd.read_csv(energy_list_path)
        self.energy_labels = self.energy_table["energy_label"].to_numpy()
        energy_ids = self.energy_table["index"].to_numpy()
        self.reference_sigmas = self.energy_table["sigma"].to_numpy()

        dvps, deps, sigs, idds = [], [], [], []
        for energy_id in energy_ids:
            lut_path = resource_filename(os.path.join(path_to_model, folder_rangeshifter_label,
                                                      "energy_%03d.csv" % energy_id))
            with open(lut_path, "r") as f:
                f.readline()  # header
                dvps.append([float(p) for p in f.readline().split(",")])
                f.readline()  # blank
                f.readline()  # header
                d, s, i = [], [], []
                for k, line in enumerate(f):
                    if k > 399:
                        break
                    parts = line.split(",")
                    d.append(float(parts[0]))
                    s.append(float(parts[1]))
                    i.append(float(parts[2]))
            deps.append(d)
            sigs.append(s)
            idds.append(i)

        self.divergence_params = np.array(dvps, dtype=np.single)
        self.lut_depths = np.array(deps, dtype=np.single)
        self.lut_sigmas = np.array(sigs, dtype=np.single)
        self.lut_idds = np.array(idds, dtype=np.single)

    def energyIDFromLabel(self, energy_label):
        energy_row = self.energy_table[self.energy_table["energy_label"] == energy_label]
        if len(energy_row) != 1:
            raise Exception("Energy ID not found for %.2f" % energy_label)
        return energy_row.index[0]


_HU_CURVES = {}

# launches of a plan's last beam in computeIMPTPlan (groups of z slabs), and
# of each other beam (splitting those too measured slower)
_TAIL_PARTS = 4
_BEAM_PARTS = 1


def _hu_curve(machine_name):
    """The machine's HU -> RLSP curve (HU_RLSP.csv), read again only when
    the file changes (the reference reads it on every call,
    plan_impt.py:158-168)."""
    path = resource_filename(os.path.join("lookuptables", "protons", machine_name,
                                          "HU_RLSP.csv"))
    st = os.stat(path)
    key = (st.st_mtime_ns, st.st_size)
    hit = _HU_CURVES.get(path)
    if hit is None or hit[0] != key:
        df = pd.read_csv(path)
        xh = df["HU"].to_numpy(dtype=np.float64)
        yh = df["RLSP"].to_numpy(dtype=np.float64)
        xh.setflags(write=False)
        yh.setflags(write=False)
        hit = _HU_CURVES[path] = (key, xh, yh)
    return hit[1], hit[2]


# Caller HU arrays seen once (address, bytes) -> weak reference, and those
# page-locked in place.
_HOST_SEEN = {}
_HOST_LOCKED = set()


def _lock_in_place(arr: np.ndarray) -> None:
    """Page-lock a caller's array in place (pb_host_register) on its second
    use, so that its upload is an asynchronous DMA from then on, as from a
    pinned tensor.  One use costs nothing extra; the lock is released when
    the array is garbage-collected.  A failure (the range overlaps one
    locked already, say) leaves the array pageable."""
    if arr.nbytes < (1 << 18) or not arr.flags.c_contiguous:
        return
    key = (arr.ctypes.data, arr.nbytes)
    if key in _HOST_LOCKED:
        return
    seen = _HOST_SEEN.get(key)
    if seen is None or seen() is not arr:
        if len(_HOST_SEEN) >= 64:   # forget arrays that are gone
            for k in [k for k, r in _HOST_SEEN.items() if r() is None]:
                del _HOST_SEEN[k]
        _HOST_SEEN[key] = weakref.ref(arr)
        return
    del _HOST_SEEN[key]
    lib = _engine()._lib
    if lib.lib.pb_host_register(ctypes.c_void_p(key[0]), key[1]) != lib.PB_OK:
        return
    _HOST_LOCKED.add(key)
    weakref.finalize(arr, _unlock, key)


def _unlock(key) -> None:
    if key in _HOST_LOCKED:
        _HOST_LOCKED.discard(key)
        try:
            _engine()._lib.lib.pb_host_unregister(ctypes.c_void_p(key[0]))
        except Exception:
            pass


def _pinned_copy(t: torch.Tensor) -> torch.Tensor:
    """An asynchronous copy of a device tensor into page-locked host memory
    (torch's pinned-memory cache), on the current stream."""
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t, non_blocking=True)
    return h


def _beam_model(plan, beam):
    try:
        model_index = list(plan.dicom_rangeshifter_label.astype(str)).index(
            beam.dicom_rangeshifter_label)
    except ValueError:
        print("Beam model not found for rangeshifter ID %s" % beam.dicom_rangeshifter_label)
        sys.exit(1)
    return plan.beam_models[model_index]


def _spot_array(beam) -> np.ndarray:
    sl = np.asarray(beam.spot_list, dtype=np.single)
    if sl.ndim == 1 and sl.size == 4:
        sl = sl.reshape(1, 4)
    if sl.ndim != 2 or (sl.size and sl.shape[1] != 4):
        raise ValueError("'spot_list' must be 2-dimensional and of type float.")
    return sl.reshape(-1, 4)


class IMPTDoseGrid(DoseGrid):

    def __init__(self):
        super().__init__()
        self.RLSP = []
        self._device_rlsp = None

    def _device(self, gpu_id):
        return _engine().require_cuda(torch.device("cuda", int(gpu_id)))

    def _check_isotropic(self):
        if self.spacing[0] != self.spacing[1] or self.spacing[0] != self.spacing[2]:
            raise Exception("Spacing must be isotropic for IMPT dose calculation - consider "
                            "resampling CT")

    def _rlsp_device(self, machine_name, device):
        # an HU array in page-locked memory goes up asynchronously; a
        # float32 array of the caller's is page-locked in place on its
        # second use
        hu_np = np.ascontiguousarray(self.HU, dtype=np.single)
        hu_h = torch.from_numpy(hu_np)
        if hu_np is self.HU and not hu_h.is_pinned():
            _lock_in_place(hu_np)
            hu_h = torch.from_numpy(hu_np)
        hu = hu_h.to(device, non_blocking=hu_h.is_pinned())
        xh, yh = _hu_curve(machine_name)
        rlsp = _engine().rlsp_from_hu(hu, xh, yh)
        self._device_rlsp = rlsp
        return rlsp

    def RLSPFromHU(self, machine_name, gpu_id=0):
        """numpy.interp of HU over the machine's HU->RLSP curve, float32
        (plan_impt.py:158-168), evaluated on the GPU."""
        rlsp = self._rlsp_device(machine_name, self._device(gpu_id))
        return rlsp.cpu().numpy().reshape(np.shape(self.HU))

    def _specs(self, plan, beams):
        specs = []
        for beam in beams:
            model = _beam_model(plan, beam)
            specs.append(_engine().BeamSpec(beam.gantry_angle, beam.couch_angle,
                                         np.asarray(beam.iso, dtype=np.single),
                                         _spot_array(beam), model))
        return specs

    def prepareIMPTPlan(self, plan, gpu_id=0, beams=None, wet_mode="texture"):
        """Device-resident plan with its WET computed: the state an
        optimisation loop reuses (engine.DevicePlan).  wet_mode "texture"
        reproduces the reference's texture-sampled WET; "exact" uses exact
        trilinear interpolation."""
        return self._prepare(plan, gpu_id, beams, wet_mode, None)

    def _prepare(self, plan, gpu_id, beams, wet_mode, pool, rlsp=None):
        self._check_isotropic()
        device = self._device(gpu_id)
        if rlsp is None:
            rlsp = self._rlsp_device(plan.machine_name, device)
        beams = plan.beam_list if beams is None else beams
        dp = _engine().DevicePlan(np.shape(self.HU), float(self.spacing[0]),
                                  np.asarray(self.origin, dtype=np.single),
                                  self._specs(plan, beams), device, texture_pool=pool)
        dp.compute_wet(rlsp.reshape(-1), wet_mode=wet_mode)
        return dp

    def _transient(self, plan, gpu_id, beams, wet_mode, rlsp=None):
        """A plan used within one call (computeIMPTPlan, computeIMPTWET): its
        texture and cell records come from this grid's pool and are kept for
        the next call."""
        pool = self.__dict__.get("_pb_texture_pool")
        if pool is None:
            pool = self._pb_texture_pool = _engine().TexturePool()
        return self._prepare(plan, gpu_id, beams, wet_mode, pool, rlsp)

    def _beam_chunks(self, plan):
        """The plan's beams in groups the device kernels take at once (the
        reference loops over any number of beams)."""
        beams = list(plan.beam_list)
        n = _engine()._lib.PB_MAX_BEAMS
        return [beams[i:i + n] for i in range(0, len(beams), n)]

    def computeIMPTPlan(self, plan, gpu_id=0, wet_mode="texture"):
        """Dose of every beam and their sum, times n_fractions
        (plan_impt.py:170-206).

        The results come back into page-locked host memory from torch's
        pinned-memory cache (reused once the previous call's arrays are
        released).  The RLSP volume's copy runs on a second stream while the
        WET and dose are computed, and the beams' doses are computed one
        beam at a time (engine.DevicePlan.forward_beam), each copied back
        while the next is computed; the plan dose is their float32 sum times
        n_fractions, as the reference forms it."""
        self.beam_doses = []
        self._check_isotropic()
        if not plan.beam_list:
            self.dose = np.zeros(self.size, dtype=np.single)
            self.RLSP = self.RLSPFromHU(plan.machine_name, gpu_id)
            self.dose *= plan.n_fractions
            return
        shape = np.shape(self.HU)
        device = self._device(gpu_id)
        main = torch.cuda.current_stream(device)
        rlsp = self._rlsp_device(plan.machine_name, device)
        side = self.__dict__.get("_pb_copy_stream")
        if side is None or side.device != device:
            # high priority: its small kernels (tile orders) start while the
            # main stream's dose kernel still has blocks waiting
            side = self._pb_copy_stream = torch.cuda.Stream(device, priority=-1)
        side.wait_stream(main)
        with torch.cuda.stream(side):
            rlsp_h = _pinned_copy(rlsp)
        chunks = self._beam_chunks(plan)
        beams_h, keep = [], []
        nf = float(plan.n_fractions)
        V = int(np.prod(shape))
        dose = torch.empty(V, dtype=torch.float32, device=device)
        dose_h = torch.empty(V, dtype=torch.float32, pin_memory=True)
        keep.append(dose)
        first_beam = True
        comp = self.__dict__.get("_pb_compute_stream")
        if comp is None or comp.device != device:
            comp = self._pb_compute_stream = torch.cuda.Stream(device)
        try:
            for chunk in chunks:
                if len(chunks) == 1:
                    # the WET is queued first; the spots are sorted into layers
                    # and uploaded on the copy stream while it runs
                    pool = self.__dict__.get("_pb_texture_pool")
                    if pool is None:
                        pool = self._pb_texture_pool = _engine().TexturePool()
                    dp = _engine().DevicePlan(shape, float(self.spacing[0]),
                                              np.asarray(self.origin, dtype=np.single),
                                              self._specs(plan, chunk), device, texture_pool=pool,
                                              defer_spots=True)
                    dp.compute_wet(rlsp.reshape(-1), check_status=False, wet_mode=wet_mode)
                    with torch.cuda.stream(side):
                        dp.load_spots()
                    main.wait_stream(side)
                else:
                    dp = self._transient(plan, gpu_id, chunk, wet_mode, rlsp)
                # One beam at a time, each in its own tile order, so that each
                # beam's dose goes back to the host while the next is computed;
                # the plan dose is the beams' float32 sum times n_fractions, as
                # the reference forms it (plan_impt.py:201-206).  The first
                # beam's tile order on the main stream, the others' (and the
                # last beam's z groups) on the copy stream while the first
                # beam's dose is computed.  The plan's last beam runs as
                # _TAIL_PARTS launches over groups of z slabs of tiles, so that
                # only the last group's doses remain to be copied back after
                # the last launch.
                nb = dp.n_beams
                final = chunk is chunks[-1]
                bd = torch.empty((nb, V), dtype=torch.float32, device=device)
                bd_h = torch.empty((nb, V), dtype=torch.float32, pin_memory=True)
                dp.beam_tile_order(0)
                side.wait_stream(main)
                with torch.cuda.stream(side):
                    launches = []
                    for b in range(nb):
                        k = _TAIL_PARTS if final and b == nb - 1 else _BEAM_PARTS
                        dp.beam_tile_order(b)
                        if k > 1:
                            launches += [(b, o, v0, v1)
                                         for o, v0, v1 in dp.beam_tile_order_parts(b, k)]
                        else:
                            launches.append((b, None, 0, V))
                    orders_ready = torch.cuda.Event()
                    orders_ready.record(side)
                # The launches alternate between two compute streams, so that a
                # launch's last blocks share the SMs with the next launch's
                # first ones; the copy stream adds each finished part into the
                # plan dose, in beam order, and copies it back.
                comp.wait_stream(main)
                for idx, (b, order, v0, v1) in enumerate(launches):
                    st = main if idx % 2 == 0 else comp
                    if idx > 0 or order is not None:
                        st.wait_event(orders_ready)
                    with torch.cuda.stream(st):
                        dp.forward_beam(b, out=bd[b], order=order)
                        done = torch.cuda.Event()
                        done.record(st)
                    side.wait_event(done)
                    last = final and b == nb - 1
                    with torch.cuda.stream(side):
                        d, db = dose[v0:v1], bd[b, v0:v1]
                        if first_beam and b == 0:
                            d.copy_(db)
                        else:
                            d.add_(db)
                        if nf != 1.0:
                            db.mul_(nf)
                            if last:
                                d.mul_(nf)
                        bd_h[b, v0:v1].copy_(db, non_blocking=True)
                        if last:
                            dose_h[v0:v1].copy_(d, non_blocking=True)
                first_beam = False
                main.wait_stream(comp)
                beams_h.append((bd_h, nb))
                keep += [bd, dp]
        except BaseException:
            # nothing queued may still use this call's buffers once they
            # are released
            for st in (main, comp, side):
                try:
                    st.synchronize()
                except Exception:
                    pass
            raise
        main.synchronize()
        side.synchronize()
        if len(chunks) == 1 and int(dp._status.item()) & _engine()._lib.PB_ERR_RAY_CAP:
            raise _engine()._lib.PbError(_engine()._lib.PB_ERR_RAY_CAP,
                                         "a WET ray reached its step cap")
        for bd_h, n in beams_h:
            arr = bd_h.numpy()
            self.beam_doses += [arr[b].reshape(shape) for b in range(n)]
        self.RLSP = rlsp_h.numpy().reshape(shape)
        self.dose = dose_h.numpy().reshape(shape)

    def computeIMPTWET(self, plan, gpu_id=0, wet_mode="texture"):
        """Per-beam WET volumes as VolumeObjects (plan_impt.py:208-236)."""
        self._check_isotropic()
        out = []
        for chunk in self._beam_chunks(plan):
            dp = self._transient(plan, gpu_id, chunk, wet_mode)
            wet = dp.wet.cpu().numpy()
            for b in range(dp.n_beams):
                wet_object = VolumeObject()
                wet_object.voxel_data = np.array(wet[b].reshape(np.shape(self.HU)),
                                                 dtype=np.single)
                wet_object.origin = np.array(self.origin, dtype=np.single)
                wet_object.spacing = np.array(self.spacing, dtype=np.single)
                out.append(wet_object)
        self.RLSP = self._device_rlsp.cpu().numpy().reshape(np.shape(self.HU))
        return out

    def computeIMPTPlanFromWET(self, plan, wet_object, beam, gpu_id=0):
        """One beam's dose from a precomputed WET volume
        (plan_impt.py:238-257); no n_fractions factor."""
        self._check_isotropic()
        device = self._device(gpu_id)
        wet = np.asarray(wet_object.voxel_data, dtype=np.single)
        dp = _engine().DevicePlan(wet.shape, float(self.spacing[0]),
                               np.asarray(self.origin, dtype=np.single),
                               self._specs(plan, [beam]), device)
        dp.set_wet(torch.from_numpy(np.ascontiguousarray(wet)).to(device))
        return dp.forward().cpu().numpy().reshape(wet.shape)

    def writeWETNRRD(self, plan, wet_path, gpu_id=0):
        if not wet_path.endswith(".nrrd"):
            raise Exception("WET path must have .nrrd extension")
        for i, w in enumerate(self.computeIMPTWET(plan, gpu_id)):
            nrrd.write(wet_path.replace(".nrrd", "_beam%02i.nrrd" % (i + 1)), w.voxel_data,
                       self.origin, self.spacing)

    def computeIMPTPlanGradient(self, plan, target_dose, voxel_weights, gpu_id=0,
                                wet_mode="texture"):
        """Quadratic objective sum_v w_v (D_v - P_v)^2 of the plan dose and its
        gradient with respect to every spot weight, in beam order then each
        beam's spot_list row order.  Returns (objective: float, gradient:
        float32 ndarray)."""
        from .autograd import plan_objective_and_grad
        chunks = self._beam_chunks(plan)
        if len(chunks) == 1:
            dp = self.prepareIMPTPlan(plan, gpu_id, wet_mode=wet_mode)
            return plan_objective_and_grad(dp, target_dose, voxel_weights,
                                           scale=float(plan.n_fractions))
        # more beams than one launch takes: the dose is the sum over the groups,
        # and each group's gradient comes from the residual of that sum
        scale = float(plan.n_fractions)
        dps = [self.prepareIMPTPlan(plan, gpu_id, beams=c, wet_mode=wet_mode) for c in chunks]
        dev = dps[0].device
        presc = torch.as_tensor(np.ascontiguousarray(target_dose, dtype=np.single),
                                device=dev).reshape(-1)
        w = torch.as_tensor(np.ascontiguousarray(voxel_weights, dtype=np.single),
                            device=dev).reshape(-1)
        dose = dps[0].forward(scale=scale)
        for dp in dps[1:]:
            dose = dose + dp.forward(scale=scale)
        resid = torch.empty_like(dose)
        obj = _engine().objective(dose, presc, w, resid)
        grads = [dp.to_plan(dp.adjoint(resid, scale=scale)).cpu().numpy() for dp in dps]
        return float(obj.item()), np.concatenate(grads)


class IMPTBeam(Beam):

    def __init__(self, beam=None):
        super().__init__()

        self.spot_list = []
        self.n_spots = 0
        self.dicom_rangeshifter_label = None

        if beam is not None:
            self.gantry_angle = beam.gantry_angle
            self.couch_angle = beam.couch_angle
            self.iso = beam.iso
            self.spot_list = beam.spot_list
            self.n_spots = beam.n_spots
            self.dicom_rangeshifter_label = beam.dicom_rangeshifter_label

    def addSpotData(self, cp, energy_id):
        """Spots of one control point (ScanSpotPositionMap, meterset weights)."""
        spm = np.reshape(np.array(cp.ScanSpotPositionMap), (-1, 2))
        mus = np.array(cp.ScanSpotMetersetWeights)
        energy_id_array = np.full(mus.size, energy_id)
        spot_list = np.array(np.column_stack((spm, mus, energy_id_array)), dtype=np.single)
        self.spot_list = np.vstack((self.spot_list, spot_list)) if self.n_spots > 0 else spot_list
        self.n_spots += mus.size

    def changeSpotEnergy(self, energy_id):
        self.spot_list[:, 3] = energy_id

    def addSingleSpot(self, x, y, mu, energy_id):
        spot = np.array([x, y, mu, energy_id], dtype=np.single)
        self.spot_list = np.vstack((self.spot_list, spot)) if self.n_spots > 0 else spot
        self.n_spots += 1

    def resetSpots(self):
        self.spot_list = np.empty((0, 4), dtype=np.single)
        self.n_spots = 0


class IMPTPlan(Plan):

    def __init__(self, machine_name="HitachiProbeatJHU"):
        super().__init__()
        self.machine_name = machine_name

        rangeshifter_list = pd.read_csv(resource_filename(os.path.join(
            "lookuptables", "protons", machine_name, "rangeshifter_labels.csv")))
        self.dicom_rangeshifter_label = rangeshifter_list["dicom_rangeshifter_label"]
        self.folder_rangeshifter_label = rangeshifter_list["folder_rangeshifter_label"]

        self.beam_models = []
        for d, f in zip(self.dicom_rangeshifter_label, self.folder_rangeshifter_label):
            self.beam_models.append(IMPTBeamModel(d, os.path.join("lookuptables", "protons",
                                                                  machine_name), f))

    def writePlanDicom(self, ct_dir, output_file, rt_struct_file=None):
        raise NotImplementedError("writePlanDicom writes DICOM through pydicom")

    def readPlanDicom(self, plan_path):
        """Beams and spots of an RT Ion Plan (plan_impt.py:635-674).

        plan_path is a file, read with pydicom (which must then be
        installed), or an RT Ion Plan dataset already read (any object with
        the DICOM attributes used below).  Per beam: the range-shifter label
        (RangeShifterSequence[0].RangeShifterID, else '0'), gantry, couch
        and isocentre from the first control point, and the spots of every
        even-numbered control point (the odd ones close each layer), with
        the energy id of its NominalBeamEnergy in the first beam model.
        The fraction count is FractionGroupSequence[0].NumberOfFractionsPlanned.
        """
        if isinstance(plan_path, (str, bytes, os.PathLike)):
            try:
                import pydicom
            except ImportError as e:
                raise ImportError("readPlanDicom needs pydicom to read a file; pass a dataset "
                                  "already read instead") from e
            ds = pydicom.dcmread(plan_path, force=True)
        else:
            ds = plan_path
        n_beams = len(ds.IonBeamSequence)
        self.n_fractions = float(ds.FractionGroupSequence[0].NumberOfFractionsPlanned)
        self.beam_list = []
        self.n_beams = 0
        for i in range(n_beams):
            ibs = ds.IonBeamSequence[i]
            beam = IMPTBeam()
            n_rs = getattr(ibs, "NumberOfRangeShifters", 0)
            if n_rs and ibs.RangeShifterSequence[0].RangeShifterID is not None:
                beam.dicom_rangeshifter_label = ibs.RangeShifterSequence[0].RangeShifterID
            else:
                beam.dicom_rangeshifter_label = '0'
            cp0 = ibs.IonControlPointSequence[0]
            beam.gantry_angle = float(cp0.GantryAngle)
            beam.couch_angle = float(cp0.PatientSupportAngle)
            beam.iso = np.array(cp0.IsocenterPosition, dtype=np.single)
            if hasattr(ibs, "BeamName"):
                beam.BeamName = ibs.BeamName
            if hasattr(ibs, "BeamDescription"):
                beam.BeamDescription = ibs.BeamDescription
            for j in range(0, len(ibs.IonControlPointSequence), 2):
                cp = ibs.IonControlPointSequence[j]
                energy_id = self.beam_models[0].energyIDFromLabel(float(cp.NominalBeamEnergy))
                beam.addSpotData(cp, energy_id)
            self.addBeam(beam)
