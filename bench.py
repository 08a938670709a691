#!/usr/bin/env python
"""Benchmark of the proton pencil-beam dose path on B200.

Workload (the differentiable plan): 256x256x160 HU at 2 mm, water with a
10 mm air margin and seeded bone/lung slabs and spheres, an ellipsoidal
target, 4 beams (0/90/180/270 deg) with ~20,000 spots on 5 mm lattices, and
the quadratic objective sum_v w_v (D_v - P_v)^2 (P = 60 in the target, 0
outside; w = 1 / 0.1).  Synthetic, seeded data (no clinical CT exists here).

Modes (the same in both arms, so that their lines compare like for like):
  forward  (default) one step = one plan's dose from its CT:
           HU -> RLSP -> WET of 4 beams -> dose.  The reference has this
           path and nothing more, so this is the step both arms time.
  grad     one step = dose + spot-weight gradient:
           HU -> RLSP -> WET -> dose -> FP64 objective + residual -> adjoint.
           The reference has no gradient: its arm prints "unavailable".
The forward line carries the dose + gradient timing too (`dose_grad`).

metric  spot-voxel evals/s = E / t_step, where E is the reference kernel's
        dense pair count sum_beams sum_layers |{v: 10 WET <= 1.1 R80}| x spots
        (the same E for every implementation, so culling counts as speed).

`value` is timed with the inputs already in HBM.  `e2e` is the same step
through the public host API: in forward mode IMPTDoseGrid.computeIMPTPlan
(host HU in, the grid's own numpy array, which that call page-locks in
place from its second use; host dose, per-beam doses and RLSP out, as the
reference's computeIMPTPlan returns them), in grad mode the library's
host-buffer optimiser step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]
                    [--mode forward|grad] [--workload plan|batch|optimize]

N > 1 runs N independent replicas (one plan per GPU, seeds differ), launched
with torch.distributed.run; the reported value is the sum over ranks of the
work divided by the slowest rank's time.  --impl reference times the
reference's own CUDA module (dose_kernels built from its sources for sm_100a
into oracle/_ref) through its host-buffer API on the same workload, driven
by a restatement of its computeIMPTPlan loop; that process loads no library
of this package (it builds the workload from the package's host-side plan
classes, which do not load libpb_b200.so).
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "dosecuda-jax_b200"), ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "IMPT dose+grad ms/plan (20k spots, 256²×160) vs plain fwd; spot-voxel evals/s"
UNIT = "spot-voxel evals/s"
L2_FLUSH_BYTES = 256 << 20
L2_NOTE = "flushed (256 MiB write) between timed iterations"
# dram__bytes_read.sum + dram__bytes_write.sum per launch, from ncu captures of
# this workload (seed 3, texture WET) on the kernels as built now; the command
# and the figures are in profiles/pencil_beam_kernels_heterogeneous_256x256x160_4beams.md.
# Reported only for that workload ("wet": k_raytrace + k_smooth).
NCU_TRAFFIC = {"k_dose_line": 208_208_128, "k_adjoint_line": 129_612_544,
               "wet": 849_633_024}
NCU_TRAFFIC_WORKLOAD = {"seed": 3, "wet_mode": "texture"}


def kernel_names():
    """Names of the forward and adjoint kernels the default shape launches."""
    from dosecuda_b200 import _lib, autotune
    name = _lib.lib.pb_dose_variant_name(autotune.default_variant()).decode()
    if autotune.shape_of(name)[0] == "l":
        return "k_dose_line", "k_adjoint_line"
    return "k_dose", "k_adjoint_tile"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(),
                                 f"pb_bench_clocks_{os.getpid()}_{index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # the sampler takes a moment to start: wait (at most 5 s) for its
        # first row, so that the rows written from here on fall inside the
        # timed region that follows
        self.skip = 0
        if self.proc is not None:
            t0 = time.time()
            while time.time() - t0 < 5.0 and self.proc.poll() is None:
                if os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.01)
            self.skip = self._rows_now()
        return self

    def _rows_now(self) -> int:
        try:
            self.f.flush()
            return len([r for r in open(self.path).read().splitlines() if r.strip()])
        except Exception:
            return 0

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r]
            # rows written during the timed region (the one before it when
            # the region was shorter than the sampling period)
            rows = rows[self.skip:] or rows[-1:]
            sm = [float(r[0]) for r in rows]
            mx = float(rows[0][1])
            reasons = sorted({names[i] for r in rows for i in range(4)
                              if r[3 + i].strip().lower() == "active"})
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons,
                    "samples": len(sm)}
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def _dist():
    from dosecuda_b200 import replicas
    return replicas.init("nccl", timeout_s=120.0)


def _barrier(world):
    from dosecuda_b200 import replicas
    replicas.barrier(world)


def _max_over_ranks(x: float, world: int, device) -> float:
    from dosecuda_b200 import replicas
    return replicas.max_over_ranks(x, world, device)


def _sum_over_ranks(x: float, world: int, device) -> float:
    from dosecuda_b200 import replicas
    return replicas.sum_over_ranks(x, world, device)


# ---------------------------------------------------------------- workload

def plan_case(seed: int):
    """The benchmarked plan (seeded), built from host-side classes only."""
    from dosecuda_b200 import phantoms
    return phantoms.config_gradient(seed=seed)


def beam_model(plan, beam):
    """The beam's model, looked up by its range-shifter label as the
    reference's computeIMPTPlan does (plan_impt.py:187-192)."""
    labels = list(plan.dicom_rangeshifter_label.astype(str))
    return plan.beam_models[labels.index(beam.dicom_rangeshifter_label)]


def spot_count(plan) -> int:
    return int(sum(np.asarray(b.spot_list).reshape(-1, 4).shape[0] for b in plan.beam_list))


def plan_config(case, mode: str) -> dict:
    """The `config` object both arms print for the plan workload."""
    g, plan = case.grid, case.plan
    nz, ny, nx = g.HU.shape
    steps = {"forward": "HU -> RLSP -> WET -> dose",
             "grad": "HU -> RLSP -> WET -> dose -> objective -> adjoint"}[mode]
    return {"workload": f"heterogeneous {nx}x{ny}x{nz} @{g.spacing[0]:g}mm, "
                        f"{len(plan.beam_list)} beams, {spot_count(plan)} spots, "
                        f"{mode} ({steps})",
            "voxels": int(nx * ny * nz), "beams": len(plan.beam_list),
            "spots": spot_count(plan), "mode": mode, "l2": L2_NOTE}


def reference_copy_bytes(case) -> tuple:
    """Bytes the reference's host API moves per plan: for each beam,
    proton_raytrace_cuda copies the RLSP volume up (its texture) and the
    smoothed WET back; proton_spot_cuda copies RLSP, WET, layers, spots,
    divergence parameters and the three LUTs up and the dose back
    (IMPTClasses.cu:274-340)."""
    g, plan = case.grid, case.plan
    V = int(np.prod(g.HU.shape))
    h2d = d2h = 0
    for beam in plan.beam_list:
        m = beam_model(plan, beam)
        sl = np.asarray(beam.spot_list).reshape(-1, 4)
        n_layers = len(np.unique(sl[:, 3]))
        n_e, lut_len = np.shape(m.lut_depths)
        h2d += 4 * V                                    # raytrace: RLSP texture
        d2h += 4 * V                                    # raytrace: WET
        h2d += 8 * V + 20 * n_layers + 16 * len(sl)     # spot: RLSP, WET, layers, spots
        h2d += 4 * n_e * (np.shape(m.divergence_params)[1] + 3 * lut_len)
        d2h += 4 * V                                    # spot: dose
    return h2d, d2h


# ------------------------------------------------------------------ mine

def run_mine(args, world, rank, local):
    import torch

    from dosecuda_b200 import engine
    from dosecuda_b200.plan_impt import _hu_curve

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    case = plan_case(args.seed + rank)
    g, plan = case.grid, case.plan
    curve = _hu_curve(plan.machine_name)
    V = int(np.prod(g.HU.shape))

    dp = g.prepareIMPTPlan(plan, local, wet_mode=args.wet_mode)
    E = dp.count_pairs()
    n_spots = dp.n_spots

    # host inputs (pinned) and their device homes
    hu_h = torch.from_numpy(np.ascontiguousarray(g.HU).reshape(-1)).pin_memory()
    presc_h = torch.from_numpy(case.presc.reshape(-1)).pin_memory()
    wts_h = torch.from_numpy(case.weights.reshape(-1)).pin_memory()
    mu_h = dp.mu_plan().cpu().pin_memory()
    hu = hu_h.to(dev)
    presc = presc_h.to(dev)
    wts = wts_h.to(dev)
    mu_plan = mu_h.to(dev)
    rlsp = torch.empty_like(hu)
    dose = torch.empty(V, dtype=torch.float32, device=dev)
    resid = torch.empty_like(dose)
    grad_sorted = torch.empty(max(n_spots, 1), dtype=torch.float32, device=dev)
    dose_out = torch.empty(V, dtype=torch.float32).pin_memory()
    grad_out = torch.empty(n_spots, dtype=torch.float32).pin_memory()
    obj_out = torch.empty(1, dtype=torch.float64).pin_memory()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    kt = {"rlsp": [], "wet": [], "order": [], "dose": [], "objective": [], "adjoint": []}

    def timed(name, fn, record):
        if record:
            a, b = ev(), ev()
            a.record(stream)
            fn()
            b.record(stream)
            kt[name].append((a, b))
        else:
            fn()

    def forward(record=False):
        timed("rlsp", lambda: engine.rlsp_from_hu(hu, *curve, out=rlsp), record)
        timed("wet", lambda: dp.compute_wet(rlsp, check_status=False, wet_mode=args.wet_mode),
              record)
        # the tile order for this WET (pb_tile_order), then the dose with it
        timed("order", dp.tile_order, record)
        timed("dose", lambda: dp.forward(dp.to_sorted(mu_plan), out=dose), record)

    obj_dev = [None]

    def step(record=False):
        forward(record)
        timed("objective", lambda: obj_dev.__setitem__(0, engine.objective(dose, presc, wts,
                                                                            resid)), record)
        timed("adjoint", lambda: dp.adjoint(resid, out=grad_sorted), record)

    # end to end through the public host API
    host_step = engine.HostGradientStep(dp, *curve, wet_mode=args.wet_mode)

    def e2e_grad():
        host_step(hu_h, presc_h, wts_h, mu_h, dose_out, grad_out, obj_out)

    # the step's input is the grid's own float32 numpy array, as a caller
    # of the reference has it; computeIMPTPlan page-locks it in place on its
    # second use (a warm-up call), so the timed calls upload it by DMA
    assert g.HU.dtype == np.float32 and g.HU.flags.c_contiguous

    def e2e_forward():
        # the reference's call: host HU in; host dose, per-beam doses and
        # RLSP out (spot sort, layer build, texture creation included)
        g.computeIMPTPlan(plan, local, wet_mode=args.wet_mode)

    def run_timed(fn, k):
        times = []
        for _ in range(k):
            flush.fill_(1.0)          # L2 flush between timed iterations
            _barrier(world)
            torch.cuda.synchronize(dev)
            a, b = ev(), ev()
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize(dev)
            times.append(a.elapsed_time(b))
        return times

    head = forward if args.mode == "forward" else step
    e2e_fn = e2e_forward if args.mode == "forward" else e2e_grad
    for _ in range(args.warmup):
        step()
        forward()
        e2e_fn()
    torch.cuda.synchronize(dev)

    with Clocks(local) as clk:
        t_head = run_timed(head, args.steps)
    t_fwd = t_head if args.mode == "forward" else run_timed(forward, args.steps)
    t_step = run_timed(lambda: step(record=True), args.steps)
    t_e2e = run_timed(e2e_fn, args.steps)
    torch.cuda.synchronize(dev)
    kms = {k: (sum(a.elapsed_time(b) for a, b in v) / len(v)) if v else None
           for k, v in kt.items()}

    ms_head = _max_over_ranks(sum(t_head) / len(t_head), world, dev)
    ms_fwd = _max_over_ranks(sum(t_fwd) / len(t_fwd), world, dev)
    ms_step = _max_over_ranks(sum(t_step) / len(t_step), world, dev)
    ms_e2e = _max_over_ranks(sum(t_e2e) / len(t_e2e), world, dev)
    E_all = _sum_over_ranks(float(E), world, dev)
    if args.mode == "forward":
        # computeIMPTPlan: the HU volume and the spot lists up; dose, every
        # beam's dose and the RLSP volume back
        h2d = 4 * V + 16 * n_spots
        d2h = 4 * V * (2 + dp.n_beams)
    else:
        h2d = 4 * (hu.numel() + presc.numel() + wts.numel() + mu_plan.numel())
        d2h = 4 * (dose.numel() + n_spots) + 8

    line = {
        "metric": METRIC,
        "value": E_all / (ms_head * 1e-3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_head,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (FP64 WET integration and objective)",
        "data": "synthetic (seeded phantom and spot plan)",
        "config": plan_config(case, args.mode),
        "dense_pairs_E": E,
        "wet_mode": args.wet_mode,
        "parallelism": f"replicas x{world}",
        "fwd_ms_per_plan": ms_fwd,
        "dose_grad": {"ms_per_plan": ms_step, "value": E_all / (ms_step * 1e-3), "unit": UNIT,
                      "over_fwd": ms_step / ms_fwd},
        "kernel_ms": kms,
        "e2e": {"value": E_all / (ms_e2e * 1e-3), "unit": UNIT, "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "call": "IMPTDoseGrid.computeIMPTPlan" if args.mode == "forward"
                else "engine.HostGradientStep"},
        # per forward step: HU->RLSP, [texture mode: five cell-record passes],
        # ray trace, smoothing, the tile order (cost, histogram, scan,
        # scatter), pencil-beam sum; the grad step adds the objective (two)
        # and the adjoint
        "gpu_launches": ((13 if args.wet_mode == "texture" else 8) +
                         (3 if args.mode == "grad" else 0)) * args.steps,
        "clocks": clk.summary(),
    }
    same = args.seed == NCU_TRAFFIC_WORKLOAD["seed"] and \
        args.wet_mode == NCU_TRAFFIC_WORKLOAD["wet_mode"]
    line.update(rooflines(dp, kms, V, E, dev, resid, NCU_TRAFFIC if same else {}))
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(case, dp, E)
    if rank == 0:
        print(json.dumps(line), flush=True)


def rooflines(dp, kms, V, E, dev, adjoint_field=None, traffic=None) -> dict:
    """Roofline lines of every kernel group over 1 ms in the step.

    HBM: algorithmic bytes per launch (each input read once, each output
    written once) over the launch's average CUDA-event time, against the
    measured copy bandwidth.  SFU: the exp2 operations the launch issues,
    counted with its own culling decisions, against the exp2 rate measured
    on this GPU now (the pencil-beam sums are exp2/FMA-issue bound, not
    traffic bound)."""
    from dosecuda_b200 import engine
    peaks, peak_kind = _peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    B, S = dp.n_beams, dp.n_spots
    lut = sum(t.dvp.numel() + 3 * t.depths.numel() for t in dp.tables) * 4
    ex2_peak = engine.measure_ex2_rate(dev)

    def hbm_line(kernel, nbytes, ms, traffic=None):
        a = nbytes / (ms * 1e-3) / 1e9
        return {"kernel": kernel, "bound": "hbm", "achieved": a, "peak": hbm, "unit": "GB/s",
                "frac": a / hbm, "peak_kind": f"of {peak_kind}",
                "algorithmic_bytes_per_launch": nbytes, "traffic": traffic}

    def sfu_line(kernel, n_ex2, n_eval, ms):
        a = n_ex2 / (ms * 1e-3)
        return {"kernel": kernel, "bound": "sfu (exp2)", "achieved": a, "peak": ex2_peak,
                "unit": "exp2/s", "frac": a / ex2_peak,
                "peak_kind": "measured now on this GPU (pb_measure_ex2_rate)",
                "exp2_per_launch": n_ex2, "spot_voxel_evaluations_per_launch": n_eval,
                "dense_pairs_E": E}

    # k_dose: WET of every beam read, dose written, per spot 32 B of geometry
    # and its weight, the LUT rows
    bytes_dose = 4 * V * (B + 1) + 36 * S + lut
    n_ex2, n_eval = dp.count_evaluated()
    k_dose, k_adj = kernel_names()
    out = {"roofline": hbm_line(f"{k_dose} (forward pencil-beam sum)", bytes_dose, kms["dose"],
                                traffic.get(k_dose)),
           "compute_roofline": sfu_line(k_dose, n_ex2, n_eval, kms["dose"])}
    lines = {}
    if kms.get("adjoint"):
        # adjoint: WET of every beam and dObj/dD read, per spot 32 B of
        # geometry and its gradient written, the LUT rows
        bytes_adj = 4 * V * (B + 1) + 36 * S + lut
        lines["adjoint"] = [hbm_line(k_adj, bytes_adj, kms["adjoint"], traffic.get(k_adj))]
        if adjoint_field is not None:
            a_ex2, a_eval = dp.count_evaluated_adjoint(adjoint_field)
            lines["adjoint"].append(sfu_line(k_adj, a_ex2, a_eval, kms["adjoint"]))
    if kms.get("wet"):
        # WET pass: RLSP read once (texture fill and cell records), raw WET
        # written and read back by the smoothing, smoothed WET written
        lines["wet"] = [hbm_line("WET (cell records + k_raytrace + k_smooth)",
                                 4 * V * (1 + 3 * B), kms["wet"], traffic.get("wet"))]
    if kms.get("rlsp"):
        lines["rlsp"] = [hbm_line("k_rlsp", 8 * V, kms["rlsp"])]
    out["kernel_rooflines"] = lines
    return out


def cpu_baseline(case, dp, E_full):
    """FP32 OpenMP port of the reference algorithm (oracle/libport32.so) on a
    bounded sample: ray trace and pencil-beam dose of all 4 beams at the
    voxels of the axial slice through the target centre."""
    from dosecuda_b200.plan_impt import _hu_curve
    from oracle import oracle as O
    g, plan = case.grid, case.plan
    shape = g.HU.shape
    nz, ny, nx = shape
    kc = int(np.argmax(case.target.sum(axis=(1, 2))))
    idx = (np.arange(ny * nx, dtype=np.int64) + kc * ny * nx)
    rlsp = O.rlsp_from_hu(g.HU, *_hu_curve(plan.machine_name))
    wet = dp.wet.cpu().numpy()
    pairs = 0
    t0 = time.perf_counter()
    for b, beam in enumerate(plan.beam_list):
        m = O.Model(beam_model(plan, beam))
        ob = O.beam_setup(beam.gantry_angle, beam.couch_angle, m.vsadx, m.vsady, beam.iso,
                          g.origin, port32=True)
        spots, layers = O.build_layers(beam.spot_list, m.dvp)
        O.raytrace(rlsp, g.spacing[0], ob, idx, port32=True)
        O.dose(wet[b].reshape(shape), g.spacing[0], ob, m, spots, layers, idx, port32=True)
        w = wet[b][idx]
        for L in layers:
            pairs += int((~(w * np.float32(10.0) > np.float32(1.1) * L["r80"])).sum()) * int(L["n_spots"])
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": pairs / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"ray trace + dense pencil-beam dose of all 4 beams at the {len(idx)} voxels "
                      f"of axial slice {kc} ({pairs} dense pairs of {E_full}); {dt:.1f} s"}


# ------------------------------------------------------------------ batch

def run_batch(args, world, rank, local):
    """Batched mode: `--batch-plans` independent plans of uneven size (grids
    64^3 .. 200x200x160 at 2-3 mm, 1-4 beams, 500-20,000 spots), WET + dose
    of all plans in one CUDA-graph replay (one batched WET launch pair and
    one persistent forward launch).  Shape chosen by the autotuner."""
    import torch

    from dosecuda_b200 import batch, phantoms

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cases = phantoms.batch_cases(seed=args.seed + 1000 * rank, n_plans=args.batch_plans)
    bp = batch.from_cases(cases, local, wet_mode=args.wet_mode)
    E = sum(dp.count_pairs() for dp in bp.plans)
    variant, bps = bp.tune()
    graph = bp.capture()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)
    times = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            _barrier(world)
            torch.cuda.synchronize(dev)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            graph.replay()
            b.record(stream)
            torch.cuda.synchronize(dev)
            times.append(a.elapsed_time(b))
    ms = _max_over_ranks(sum(times) / len(times), world, dev)
    E_all = _sum_over_ranks(float(E), world, dev)
    from dosecuda_b200 import autotune
    line = {
        "metric": "IMPT batched forward (WET + dose of every plan, one CUDA-graph replay); "
                  "spot-voxel evals/s",
        "value": E_all / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (FP64 WET integration)", "data": "synthetic",
        "config": {"workload": f"{bp.n_plans} uneven plans per GPU",
                   "voxels": bp.n_vox, "spots": bp.n_spots, "tiles": bp.n_tiles,
                   "dense_pairs_E": E, "wet_mode": args.wet_mode,
                   "variant": autotune.variants()[variant], "blocks_per_sm": bps,
                   "plans_per_s": bp.n_plans * world / (ms * 1e-3),
                   "l2": L2_NOTE},
        "gpu_launches": 4 * args.steps,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


# -------------------------------------------------------------- optimise

def run_optimize(args, world, rank, local):
    """Large optimisation loop: 512x512x200 at 1 mm, 4 beams, ~60,000 spots;
    `--opt-iters` projected-gradient iterations (forward + FP64 objective +
    adjoint + projection) replayed from one CUDA graph, WET computed once and
    kept on the device; the final dose is checked against the FP64 oracle at
    sampled voxels."""
    import torch

    from dosecuda_b200 import optimize, phantoms

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    case = phantoms.config_optimisation(seed=args.seed + rank)
    g, plan = case.grid, case.plan
    dp = g.prepareIMPTPlan(plan, local, wet_mode=args.wet_mode)
    E = dp.count_pairs()
    opt = optimize.ProjectedGradient(dp, torch.from_numpy(case.presc),
                                     torch.from_numpy(case.weights),
                                     scale=float(plan.n_fractions))
    opt.prepare()
    opt.run(args.warmup)
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    _barrier(world)
    with Clocks(local) as clk:
        a.record(stream)
        hist = opt.run(args.opt_iters)
        b.record(stream)
        torch.cuda.synchronize(dev)
    ms_total = _max_over_ranks(a.elapsed_time(b), world, dev)
    ms_iter = ms_total / args.opt_iters
    E_all = _sum_over_ranks(float(E), world, dev)
    hist = hist.cpu().numpy()
    check = {}
    if rank == 0 and not args.no_cpu_baseline:
        check = _oracle_check(case, dp, opt)
    line = {
        "metric": "IMPT projected-gradient iterations (512x512x200 @1mm, 4 beams, ~60k spots); "
                  "spot-voxel evals/s",
        "value": E_all / (ms_iter * 1e-3), "unit": UNIT, "n_gpus": world,
        "steps": args.opt_iters, "warmup": args.warmup, "ms_per_step": ms_iter,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (FP64 WET integration and objective)", "data": "synthetic",
        "config": {"workload": "optimisation loop, 512x512x200 @1mm, 4 beams, "
                               f"{dp.n_spots} spots", "voxels": dp.n_vox,
                   "dense_pairs_E": E, "iterations": args.opt_iters,
                   "loop_ms": ms_total, "step_eta": opt.eta,
                   "objective_first": float(hist[0]), "objective_last": float(hist[-1]),
                   "objective_monotone": bool((hist[1:] <= hist[:-1] * (1 + 1e-9)).all()),
                   "wet_mode": args.wet_mode},
        "final_dose_vs_fp64_oracle": check,
        "gpu_launches": 6 * args.opt_iters,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def _oracle_check(case, dp, opt, n_random=600):
    """Final dose at the 400 hottest and `n_random` random voxels vs the FP64
    oracle on the same WET and weights: max |D - D_oracle| / Dmax."""
    from oracle import oracle as O
    g, plan = case.grid, case.plan
    dose = opt.final_dose().cpu().numpy()
    wet = dp.wet.cpu().numpy()
    mu = opt.mu_plan().cpu().numpy()
    rng = np.random.default_rng(0)
    idx = np.unique(np.concatenate([np.argsort(dose)[-400:],
                                    rng.choice(dose.size, n_random, replace=False)]))
    want = np.zeros(len(idx))
    row = 0
    for b, beam in enumerate(plan.beam_list):
        sl = np.asarray(beam.spot_list, np.float32).reshape(-1, 4).copy()
        sl[:, 2] = mu[row: row + len(sl)]
        row += len(sl)
        m = O.Model(beam_model(plan, beam))
        ob = O.beam_setup(beam.gantry_angle, beam.couch_angle, m.vsadx, m.vsady, beam.iso,
                          g.origin)
        spots, layers = O.build_layers(sl, m.dvp)
        want += O.dose(wet[b].reshape(g.HU.shape), g.spacing[0], ob, m, spots, layers,
                       idx.astype(np.int64))
    want *= float(plan.n_fractions)
    dmax = float(dose.max())
    return {"voxels": int(len(idx)), "max_abs_err_over_dmax":
            float(np.abs(dose[idx] - want).max() / dmax), "dmax": dmax}


# -------------------------------------------------------------- reference

def _unavailable(why: str) -> None:
    print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)


def load_reference_module():
    """The reference's dose_kernels module built from its sources into
    oracle/_ref, or None."""
    paths = glob.glob(os.path.join(ROOT, "oracle", "_ref", "dose_kernels*.so"))
    if not paths:
        return None
    import importlib.machinery
    import importlib.util
    loader = importlib.machinery.ExtensionFileLoader("dose_kernels", paths[0])
    spec = importlib.util.spec_from_file_location("dose_kernels", paths[0], loader=loader)
    ref = importlib.util.module_from_spec(spec)
    loader.exec_module(ref)
    return ref


def run_reference(args, world, rank, local):
    """The reference's CUDA module on this GPU, driven as its
    computeIMPTPlan drives it (plan_impt.py:170-206): host numpy HU -> RLSP,
    then per beam proton_raytrace_cuda and proton_spot_cuda (each with its
    own device allocation and host copies), the beam doses summed on the
    host and scaled by n_fractions.  Nothing of this package's device code
    is loaded in this process."""
    if rank != 0:
        return
    if args.workload != "plan":
        _unavailable(f"the reference has no {args.workload} mode (one beam of one plan per call)")
        return
    if args.mode != "forward":
        _unavailable("the reference has no gradient: only its forward dose can be timed")
        return
    ref = load_reference_module()
    if ref is None:
        _unavailable("oracle/_ref/dose_kernels was not built (needs the reference sources)")
        return
    import torch

    from dosecuda_b200.plan import VolumeObject
    from dosecuda_b200.plan_impt import _hu_curve
    from oracle import oracle as O

    torch.cuda.set_device(local)
    case = plan_case(args.seed)
    g, plan = case.grid, case.plan
    curve = _hu_curve(plan.machine_name)

    def vol(data):
        v = VolumeObject()
        v.voxel_data = data
        v.origin = np.array(g.origin, dtype=np.single)
        v.spacing = np.array(g.spacing, dtype=np.single)
        return v

    for b in plan.beam_list:
        b.spot_list = np.asarray(b.spot_list, np.float32).reshape(-1, 4)
    wets = []

    def step():
        rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
        dose = np.zeros(g.HU.shape, dtype=np.single)
        beam_doses = []
        wets.clear()
        for beam in plan.beam_list:
            model = beam_model(plan, beam)
            w = ref.proton_raytrace_cuda(model, vol(rlsp), beam, local)
            wets.append(w)
            d = ref.proton_spot_cuda(model, vol(rlsp), vol(w), beam, local)
            beam_doses.append(d * plan.n_fractions)
            dose += d
        dose *= plan.n_fractions
        return dose

    dev = torch.device("cuda", local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        step()
    E = 0
    for b, beam in enumerate(plan.beam_list):
        _, layers = O.build_layers(beam.spot_list, beam_model(plan, beam).divergence_params)
        E += O.count_pairs(wets[b], layers)
    times = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()           # synchronous: returns after the dose copy
            b.record(stream)
            torch.cuda.synchronize(dev)
            times.append(a.elapsed_time(b))
    ms = sum(times) / len(times)
    value = E / (ms * 1e-3)
    h2d, d2h = reference_copy_bytes(case)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": plan_config(case, args.mode),
        "dense_pairs_E": E,
        "parallelism": "one process (rank 0)",
        "e2e": {"value": value, "unit": UNIT, "ms_per_step": ms, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "call": "computeIMPTPlan loop over dose_kernels"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "runs_on": "gpu",
                         "sample": "the whole workload, every step.  The reference's path is "
                                   "CUDA: this is its dose_kernels module on this B200, driven "
                                   "from one host thread through its host-buffer API (host numpy "
                                   "HU->RLSP, per-beam device allocation and copies); its JAX "
                                   "CPU path cannot run here (no jax)"},
        "clocks": clk.summary(),
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--mode", choices=["forward", "grad"], default="forward")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--wet-mode", choices=["texture", "exact"], default="texture")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["plan", "batch", "optimize"], default="plan")
    ap.add_argument("--opt-iters", type=int, default=50)
    ap.add_argument("--batch-plans", type=int, default=32)
    args = ap.parse_args()
    if args.impl == "reference":
        # one process times the reference; other ranks of a multi-GPU launch
        # exit without work and without joining a process group
        rank = int(os.environ.get("RANK", "0"))
        if rank == 0:
            run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), 0,
                          int(os.environ.get("LOCAL_RANK", "0")))
        return
    world, rank, local = _dist()
    try:
        if args.workload == "batch":
            run_batch(args, world, rank, local)
        elif args.workload == "optimize":
            run_optimize(args, world, rank, local)
        else:
            run_mine(args, world, rank, local)
    finally:
        from dosecuda_b200 import replicas
        replicas.finish(world)


if __name__ == "__main__":
    main()
