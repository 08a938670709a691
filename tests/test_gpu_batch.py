"""Batched multi-plan mode and the autotuner, on the GPU.

The batch runs every (plan, beam) WET in one launch and every plan's
forward dose in one persistent launch; each voxel's arithmetic is the same
as in the single-plan kernels, so results are compared for equality."""
import numpy as np
import pytest
import torch

from conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def cases():
    from dosecuda_b200 import phantoms
    return phantoms.batch_cases(seed=11, n_plans=5, min_shape=(24, 24, 24),
                                max_shape=(40, 44, 52), spacings=(3.0, 4.0), spots=(100, 500))


@pytest.mark.parametrize("wet_mode", ["texture", "exact"])
def test_batch_matches_single_plans(cases, wet_mode):
    from dosecuda_b200 import batch
    bp = batch.from_cases(cases, 0, wet_mode=wet_mode)
    single_wet = [dp.wet.clone() for dp in bp.plans]
    single = [dp.forward() for dp in bp.plans]
    for dp in bp.plans:
        dp.wet.zero_()
    bp.run()
    torch.cuda.synchronize()
    assert int(bp.status.item()) == 0
    for p, dp in enumerate(bp.plans):
        assert torch.equal(dp.wet, single_wet[p])
        assert torch.equal(bp.doses[p], single[p])
        assert float(single[p].max()) > 0


def test_forward_variants_agree(cases):
    dp = cases[0].grid.prepareIMPTPlan(cases[0].plan, 0)
    ref = dp.forward()
    from dosecuda_b200 import autotune
    for v in range(len(autotune.variants())):
        assert torch.equal(dp.forward_variant(v), ref), v


def test_batch_variants_and_grids_agree(cases):
    from dosecuda_b200 import autotune, batch
    bp = batch.from_cases(cases, 0)
    bp.run()
    ref = [d.clone() for d in bp.doses]
    for v, bps in autotune.batch_candidates()[::3]:
        for d in bp.doses:
            d.zero_()
        bp.run(variant=v, blocks_per_sm=bps)
        for p in range(bp.n_plans):
            assert torch.equal(bp.doses[p], ref[p]), (v, bps, p)


def test_batch_graph_replay_reads_new_weights(cases):
    from dosecuda_b200 import batch
    bp = batch.from_cases(cases, 0)
    graph = bp.capture()
    graph.replay()
    torch.cuda.synchronize()
    base = [d.clone() for d in bp.doses]
    mu0 = bp.plans[0].mu_plan()
    bp.set_mu(0, mu0 * 2.0)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.allclose(bp.doses[0], 2.0 * base[0], rtol=1e-5,
                          atol=1e-6 * float(base[0].max()))
    for p in range(1, bp.n_plans):
        assert torch.equal(bp.doses[p], base[p])
    bp.set_mu(0, mu0)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(bp.doses[0], base[0])


def test_autotuner_picks_and_caches(cases, tmp_path, monkeypatch):
    from dosecuda_b200 import autotune, batch
    monkeypatch.setenv("DOSECUDA_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    dp = cases[1].grid.prepareIMPTPlan(cases[1].plan, 0)
    v = autotune.tune_plan(dp, reps=1)
    assert 0 <= v < len(autotune.variants())
    assert autotune.tune_plan(dp, reps=1) == v            # from the cache
    bp = batch.from_cases(cases[:3], 0)
    v2, bps = bp.tune()
    assert (v2, bps) in autotune.batch_candidates()
    assert (tmp_path / "tune.json").exists()
