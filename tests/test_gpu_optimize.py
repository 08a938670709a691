"""Projected gradient descent on the GPU: monotone objective, feasible
weights, graph replay equal to eager steps."""
import numpy as np
import pytest
import torch

from conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _problem():
    from dosecuda_b200 import phantoms
    c = phantoms.small_heterogeneous(seed=21)
    dp = c.grid.prepareIMPTPlan(c.plan, 0)
    return c, dp


def test_pgd_decreases_objective_and_keeps_weights_feasible():
    from dosecuda_b200 import optimize
    c, dp = _problem()
    opt = optimize.ProjectedGradient(dp, torch.from_numpy(c.presc), torch.from_numpy(c.weights))
    opt.prepare()
    hist = opt.run(15).cpu().numpy()
    assert np.all(np.diff(hist) <= 1e-9 * hist[0])
    assert hist[-1] < 0.9 * hist[0]
    assert float(opt.mu.min()) >= 0.0


def test_graph_replay_equals_eager_steps():
    from dosecuda_b200 import optimize
    c, dp = _problem()
    a = optimize.ProjectedGradient(dp, torch.from_numpy(c.presc), torch.from_numpy(c.weights))
    a.prepare(capture=True)
    b = optimize.ProjectedGradient(dp, torch.from_numpy(c.presc), torch.from_numpy(c.weights))
    b.eta = a.eta
    b.mu.copy_(a.mu)              # a.prepare ran one warm-up step
    ha = a.run(4).cpu().numpy()
    hb = np.array([0.0] * 4)
    for i in range(4):
        b.step()
        hb[i] = float(b.obj.item())
    assert np.allclose(ha, hb, rtol=1e-6)
    assert torch.allclose(a.mu, b.mu, rtol=1e-5, atol=1e-6)
