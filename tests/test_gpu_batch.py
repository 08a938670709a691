"""Batched multi-plan mode and the autotuner, on the GPU.

The batch runs every (plan, beam) WET in one launch and every plan's
forward dose in one persistent launch; each voxel's arithmetic is the same
as in the single-plan kernel of the same shape, so results are compared for
equality.  Kernel shapes that cull a different number of spots per round
add a layer's spots in a different order when the layer has more spots
than a round: those agree to rounding."""
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
    single = [dp.forward_variant(bp.variant) for dp in bp.plans]
    for dp in bp.plans:
        dp.wet.zero_()
    bp.run()
    torch.cuda.synchronize()
    assert int(bp.status.item()) == 0
    for p, dp in enumerate(bp.plans):
        assert torch.equal(dp.wet, single_wet[p])
        assert torch.equal(bp.doses[p], single[p])
        assert float(single[p].max()) > 0


def _same_decisions(a, b):
    """Shapes whose doses are equal bit for bit (same family, tile and
    round size); other shapes agree to rounding."""
    from dosecuda_b200 import autotune
    return autotune.same_decisions(a, b)


@pytest.mark.parametrize("pitch", [5.0, 1.5])
def test_forward_variants_agree(pitch):
    """Every kernel shape gives the default's dose: bit for bit with the same
    family, tile and round size, to rounding otherwise (other tiles cull
    differently; on the 1.5 mm lattice a layer holds ~240 spots, more than
    some shapes' rounds)."""
    from dosecuda_b200 import autotune, phantoms
    case = phantoms.heterogeneous(7, (0.0, 135.0), 4000, shape=(40, 48, 56), spacing=3.0,
                                  n_slabs=1, n_spheres=2, semi_range=(10.0, 16.0),
                                  centre_jitter=5.0, body_inset=15.0, pitch=pitch)
    dp = case.grid.prepareIMPTPlan(case.plan, 0)
    ref = dp.forward()
    names = autotune.variants()
    dflt = names[autotune.default_variant()]
    for v, name in enumerate(names):
        d = dp.forward_variant(v)
        if _same_decisions(name, dflt):
            assert torch.equal(d, ref), name
        else:
            # the two families form the axis distance by different FP32
            # operation orders: agreement to a few units of rounding
            assert torch.allclose(d, ref, rtol=1e-5, atol=1e-5 * float(ref.max())), name


def test_adjoint_families_agree():
    """The spot-weight gradient of each kernel family on the same residual:
    equal to float rounding (1e-5 of max |g|)."""
    from dosecuda_b200 import autotune, phantoms
    case = phantoms.small_heterogeneous(seed=19)
    dp = case.grid.prepareIMPTPlan(case.plan, 0)
    w = torch.from_numpy(np.random.default_rng(2).normal(size=dp.n_vox).astype(np.float32))
    w = w.to(dp.device)
    names = autotune.variants()
    fams = {}
    for v, name in enumerate(names):
        fams.setdefault(autotune.shape_of(name)[0], v)
    assert set(fams) == {"t", "l"}
    g = {f: dp.adjoint(w, variant=v).clone() for f, v in fams.items()}
    m = float(g["t"].abs().max())
    assert m > 0 and float((g["l"] - g["t"]).abs().max()) <= 1e-5 * m
    # the default adjoint is the line family's (its cross-tile sums are
    # float atomics, so only to rounding)
    assert float((dp.adjoint(w) - g["l"]).abs().max()) <= 1e-5 * m


def test_batch_variants_and_grids_agree(cases):
    from dosecuda_b200 import autotune, batch
    bp = batch.from_cases(cases, 0)
    bp.run()
    ref = [d.clone() for d in bp.doses]
    names = autotune.variants()
    for v, bps in autotune.batch_candidates()[::3]:
        for d in bp.doses:
            d.zero_()
        bp.run(variant=v, blocks_per_sm=bps)
        for p in range(bp.n_plans):
            if _same_decisions(names[v], names[bp.variant]):
                assert torch.equal(bp.doses[p], ref[p]), (v, bps, p)
            else:
                assert torch.allclose(bp.doses[p], ref[p], rtol=1e-5,
                                      atol=1e-6 * float(ref[p].max())), (v, bps, p)


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
