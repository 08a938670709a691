#!/usr/bin/env python
"""Benchmark of the proton pencil-beam dose path on B200.

Workload (the differentiable plan): 256x256x160 HU at 2 mm, water with a
10 mm air margin and seeded bone/lung slabs and spheres, an ellipsoidal
target, 4 beams (0/90/180/270 deg) with ~20,000 spots on 5 mm lattices, and
the quadratic objective sum_v w_v (D_v - P_v)^2 (P = 60 in the target, 0
outside; w = 1 / 0.1).  Synthetic, seeded data (no clinical CT exists here).

One step = one plan evaluation with its spot-weight gradient:
    HU -> RLSP -> WET of 4 beams -> forward dose -> FP64 objective + residual
    -> adjoint (d objective / d spot weight)
The plain forward (HU -> RLSP -> WET -> dose) is timed beside it.

metric  spot-voxel evals/s = E / t_step, where E is the reference kernel's
        dense pair count sum_beams sum_layers |{v: 10 WET <= 1.1 R80}| x spots
        (the same E for every implementation, so culling counts as speed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

N > 1 runs N independent replicas (one plan per GPU, seeds differ), launched
with torch.distributed.run; the reported value is the sum over ranks of the
work divided by the slowest rank's time.  --impl reference times the
reference's own CUDA module (dose_kernels built from its sources for sm_100a
into oracle/_ref) through its host-buffer API on the same workload; it has
no gradient, so its step is the plain forward.
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
# dram__bytes_read.sum + dram__bytes_write.sum of one k_dose launch of the
# default workload (seed 3, texture WET), from the ncu --set full capture
# summarised in profiles/pencil_beam_kernels_heterogeneous_256x256x160_4beams.md
K_DOSE_TRAFFIC = 169_035_520 + 32_191_488


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


# ------------------------------------------------------------------ mine

def run_mine(args, world, rank, local):
    import torch

    from dosecuda_b200 import engine, phantoms
    from dosecuda_b200.plan_impt import _hu_curve

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    case = phantoms.config_gradient(seed=args.seed + rank)
    g, plan = case.grid, case.plan
    curve = _hu_curve(plan.machine_name)
    shape = g.HU.shape
    V = int(np.prod(shape))

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
    kt = {"rlsp": [], "wet": [], "dose": [], "objective": [], "adjoint": []}

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
        timed("dose", lambda: dp.forward(dp.to_sorted(mu_plan), out=dose), record)

    obj_dev = [None]

    def step(record=False):
        forward(record)
        timed("objective", lambda: obj_dev.__setitem__(0, engine.objective(dose, presc, wts,
                                                                            resid)), record)
        timed("adjoint", lambda: dp.adjoint(resid, out=grad_sorted), record)

    # end to end: the library's host-buffer step (inputs up from pinned host
    # memory, dose / gradient / objective back), copies overlapped with the
    # kernels where they are off the critical path
    host_step = engine.HostGradientStep(dp, *curve, wet_mode=args.wet_mode)

    def e2e_step():
        host_step(hu_h, presc_h, wts_h, mu_h, dose_out, grad_out, obj_out)

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

    for _ in range(args.warmup):
        step()
        forward()
        e2e_step()
    torch.cuda.synchronize(dev)

    with Clocks(local) as clk:
        t_step = run_timed(lambda: step(record=True), args.steps)
    t_fwd = run_timed(forward, args.steps)
    t_e2e = run_timed(e2e_step, args.steps)
    torch.cuda.synchronize(dev)
    kms = {k: (sum(a.elapsed_time(b) for a, b in v) / len(v)) if v else None
           for k, v in kt.items()}

    ms_step = _max_over_ranks(sum(t_step) / len(t_step), world, dev)
    ms_fwd = _max_over_ranks(sum(t_fwd) / len(t_fwd), world, dev)
    ms_e2e = _max_over_ranks(sum(t_e2e) / len(t_e2e), world, dev)
    E_all = _sum_over_ranks(float(E), world, dev)
    h2d = 4 * (hu.numel() + presc.numel() + wts.numel() + mu_plan.numel())
    d2h = 4 * (dose.numel() + n_spots) + 8

    peaks, peak_kind = _peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    # dominant kernel: the forward pencil-beam kernel (k_dose, one launch per step)
    bytes_dose = 4 * V * (dp.n_beams + 1) + 36 * n_spots + \
        sum(t.dvp.numel() + 3 * t.depths.numel() for t in dp.tables) * 4
    achieved = bytes_dose / (kms["dose"] * 1e-3) / 1e9
    # SFU roofline of the same kernel: the exp2 operations one launch issues
    # (counted with its own culling decisions) over its time, against the
    # exp2 throughput measured on this GPU now
    n_ex2, n_eval = dp.count_evaluated()
    ex2_peak = engine.measure_ex2_rate(dev)
    ex2_achieved = n_ex2 / (kms["dose"] * 1e-3)
    # DRAM traffic of one k_dose launch from the ncu capture of this workload
    traffic = K_DOSE_TRAFFIC if (args.seed == 3 and args.wet_mode == "texture") else None
    line = {
        "metric": METRIC,
        "value": E_all / (ms_step * 1e-3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (FP64 WET integration and objective)",
        "data": "synthetic (seeded phantom and spot plan)",
        "config": {"workload": "heterogeneous 256x256x160 @2mm, 4 beams, "
                               f"{n_spots} spots, quadratic objective (dose+grad)",
                   "voxels": V, "beams": dp.n_beams, "spots": n_spots,
                   "dense_pairs_E": E, "wet_mode": args.wet_mode,
                   "l2": "flushed (256 MiB write) between timed iterations",
                   "parallelism": f"replicas x{world}"},
        "fwd_ms_per_plan": ms_fwd,
        "dose_grad_over_fwd": ms_step / ms_fwd,
        "kernel_ms": kms,
        "e2e": {"value": E_all / (ms_e2e * 1e-3), "unit": UNIT, "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        # per step: HU->RLSP, [texture mode: five cell-record passes], ray trace,
        # smoothing, pencil-beam sum, objective (two), adjoint
        "gpu_launches": (12 if args.wet_mode == "texture" else 7) * args.steps,
        "roofline": {"kernel": "k_dose (forward pencil-beam sum)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": f"of {peak_kind}",
                     "algorithmic_bytes_per_launch": bytes_dose, "traffic": traffic},
        "compute_roofline": {"kernel": "k_dose", "bound": "sfu (exp2)",
                             "achieved": ex2_achieved, "peak": ex2_peak, "unit": "exp2/s",
                             "frac": ex2_achieved / ex2_peak,
                             "peak_kind": "measured now on this GPU (pb_measure_ex2_rate)",
                             "exp2_per_launch": n_ex2,
                             "spot_voxel_evaluations_per_launch": n_eval,
                             "dense_pairs_E": E},
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(case, dp, E)
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_baseline(case, dp, E_full):
    """FP32 OpenMP port of the reference algorithm (oracle/libport32.so) on a
    bounded sample: ray trace and pencil-beam dose of all 4 beams at the
    voxels of the axial slice through the target centre."""
    from oracle import oracle as O
    g, plan = case.grid, case.plan
    shape = g.HU.shape
    nz, ny, nx = shape
    kc = int(np.argmax(case.target.sum(axis=(1, 2))))
    idx = (np.arange(ny * nx, dtype=np.int64) + kc * ny * nx)
    rlsp = O.rlsp_from_hu(g.HU, *__import__("dosecuda_b200.plan_impt", fromlist=["x"])._hu_curve(
        plan.machine_name))
    wet = dp.wet.cpu().numpy()
    pairs = 0
    t0 = time.perf_counter()
    for b, beam in enumerate(plan.beam_list):
        m = O.Model(plan.beam_models[0])
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
                   "l2": "flushed (256 MiB write) between timed iterations"},
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
        m = O.Model(plan.beam_models[0])
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

def run_reference(args, world, rank, local):
    if rank != 0:
        return
    import torch

    from dosecuda_b200 import phantoms
    from dosecuda_b200.plan import VolumeObject
    from dosecuda_b200.plan_impt import _hu_curve
    from oracle import oracle as O
    paths = glob.glob(os.path.join(ROOT, "oracle", "_ref", "dose_kernels*.so"))
    if not paths:
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/dose_kernels was not built (needs the reference sources)"}))
        return
    import importlib.machinery
    import importlib.util
    loader = importlib.machinery.ExtensionFileLoader("dose_kernels", paths[0])
    spec = importlib.util.spec_from_file_location("dose_kernels", paths[0], loader=loader)
    ref = importlib.util.module_from_spec(spec)
    loader.exec_module(ref)

    case = phantoms.config_gradient(seed=args.seed)
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
        # computeIMPTPlan's loop (plan_impt.py:170-206) on the reference module
        rlsp = np.array(np.interp(g.HU, *curve), dtype=np.single)
        dose = np.zeros(g.HU.shape, dtype=np.single)
        wets.clear()
        for beam in plan.beam_list:
            w = ref.proton_raytrace_cuda(plan.beam_models[0], vol(rlsp), beam, local)
            wets.append(w)
            dose += ref.proton_spot_cuda(plan.beam_models[0], vol(rlsp), vol(w), beam, local)
        dose *= plan.n_fractions
        return dose

    for _ in range(args.warmup):
        step()
    E = 0
    for b, beam in enumerate(plan.beam_list):
        _, layers = O.build_layers(beam.spot_list, plan.beam_models[0].divergence_params)
        E += O.count_pairs(wets[b], layers)
    times = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            step()
            torch.cuda.synchronize()
            times.append((time.perf_counter() - t0) * 1e3)
    ms = sum(times) / len(times)
    value = E / (ms * 1e-3)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "heterogeneous 256x256x160 @2mm, 4 beams, "
                               f"{sum(len(b.spot_list) for b in plan.beam_list)} spots "
                               "(plain forward: the reference has no gradient)",
                   "dense_pairs_E": E},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "the whole workload; the reference's path is CUDA: its "
                                   "dose_kernels module built from its sources for sm_100a, "
                                   "driven from one host thread through its host-buffer API "
                                   "(host numpy HU->RLSP, per-beam device allocation and copies)"},
        "clocks": clk.summary(),
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--wet-mode", choices=["texture", "exact"], default="texture")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["gradient", "batch", "optimize"], default="gradient")
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
