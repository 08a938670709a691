"""Many plans in one launch: the batched WET pass and the persistent
forward dose kernel (pb_batch_setup / pb_batch_run), capturable once as a
CUDA graph and replayed.

Each plan keeps its own grid, beams, spots and model tables (prepared as an
``engine.DevicePlan``); the batch adds only its device records and a work
queue.  Plans may differ in grid size, spacing, beam count and spot count.
The reference computes one beam of one plan per call
(DoseCUDA/plan_impt.py:185-206, IMPTClasses.cu:274-340).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import torch

from . import _lib, autotune, engine
from ._lib import check, ptr


class BatchPlans:
    """A fixed batch of plans resident on one GPU."""

    def __init__(self, plans: Sequence["engine.DevicePlan"], rlsps: Sequence[torch.Tensor],
                 scales: Optional[Sequence[float]] = None):
        if not plans:
            raise ValueError("a batch needs at least one plan")
        self.plans: List[engine.DevicePlan] = list(plans)
        self.device = self.plans[0].device
        for dp in self.plans:
            if dp.device != self.device:
                raise ValueError("all plans of a batch must live on one device")
            dp._need_wet()
        self.n_plans = len(self.plans)
        self.n_vox = sum(dp.n_vox for dp in self.plans)
        self.n_spots = sum(dp.n_spots for dp in self.plans)
        self.rlsps = [r.contiguous() for r in rlsps]
        scales = [1.0] * self.n_plans if scales is None else list(scales)
        self.doses = [torch.zeros(dp.n_vox, dtype=torch.float32, device=self.device)
                      for dp in self.plans]
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        recs = (_lib.PbBatchPlan * self.n_plans)()
        for p, dp in enumerate(self.plans):
            R = recs[p]
            R.grid = dp.grid
            R.n_beams = dp.n_beams
            for b in range(dp.n_beams):
                R.beams[b] = dp.beams[b]
            R.rlsp_dev = self.rlsps[p].data_ptr()
            # the handle of the plan's last WET mode: texture, or the exact
            # mode's cell records
            R.tex = dp._tex.value if dp.wet_mode == "texture" else dp._cells.value
            R.raw_work_dev = dp.raw_wet.data_ptr()
            R.wet_dev = dp.wet.data_ptr()
            R.layers_dev = dp.layers.data_ptr()
            R.spot_geo_dev = dp.spot_geo.data_ptr()
            R.mu_dev = dp.mu_sorted.data_ptr()
            R.scale = float(scales[p])
            R.dose_dev = self.doses[p].data_ptr()
        self._recs = recs
        self.work = torch.zeros(int(_lib.lib.pb_batch_work_size(self.n_plans)), dtype=torch.uint8,
                                device=self.device)
        self.info = _lib.PbBatchInfo()
        check(_lib.lib.pb_batch_setup(ctypes.cast(recs, ctypes.c_void_p), self.n_plans,
                                      ptr(self.work), ctypes.byref(self.info),
                                      engine._stream(self.device)), "pb_batch_setup")
        self.variant = autotune.default_batch_variant()
        self.blocks_per_sm = 4

    @property
    def n_tiles(self) -> int:
        return int(self.info.n_tiles)

    def tune(self, use_cache: bool = True):
        """Pick the forward shape and persistent grid with the autotuner."""
        self.variant, self.blocks_per_sm = autotune.tune_batch(self, use_cache=use_cache)
        return self.variant, self.blocks_per_sm

    def run(self, flags: int = _lib.PB_BATCH_WET | _lib.PB_BATCH_DOSE,
            variant: Optional[int] = None, blocks_per_sm: Optional[int] = None) -> None:
        """Stream-ordered run of the batch (no host synchronisation)."""
        check(_lib.lib.pb_batch_run(ctypes.byref(self.info), ptr(self.work), int(flags),
                                    self.variant if variant is None else int(variant),
                                    self.blocks_per_sm if blocks_per_sm is None
                                    else int(blocks_per_sm),
                                    ptr(self.status), engine._stream(self.device)),
              "pb_batch_run")

    def capture(self, flags: int = _lib.PB_BATCH_WET | _lib.PB_BATCH_DOSE) -> torch.cuda.CUDAGraph:
        """Capture one run of the batch in a CUDA graph (replay with .replay())."""
        self.run(flags)              # warm-up outside the capture
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.run(flags)
        return graph

    def set_mu(self, p: int, mu_plan: torch.Tensor) -> None:
        """Overwrite plan p's spot weights in place (plan row order); a
        captured graph reads the new values at its next replay."""
        dp = self.plans[p]
        dp.mu_sorted.copy_(dp.to_sorted(mu_plan.to(self.device, torch.float32)))


def from_cases(cases, gpu_id: int = 0, wet_mode: str = "texture") -> BatchPlans:
    """Batch of phantoms.SynthCase-like cases (grid, plan), n_fractions as scale."""
    plans, rlsps, scales = [], [], []
    for c in cases:
        dp = c.grid.prepareIMPTPlan(c.plan, gpu_id, wet_mode=wet_mode)
        plans.append(dp)
        rlsps.append(c.grid._device_rlsp.reshape(-1))
        scales.append(float(c.plan.n_fractions))
    return BatchPlans(plans, rlsps, scales)
