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


def test_host_step_equals_device_step_twice():
    """The host-buffer step (copies overlapped on a second stream) gives the
    device-resident step's dose and objective bit for bit, and its gradient
    up to the order of the adjoint's atomic sums (1e-5 of max |g|), on two
    steps in a row with different spot weights."""
    from dosecuda_b200 import engine
    from dosecuda_b200.plan_impt import _hu_curve
    c, dp = _problem()
    curve = _hu_curve(c.plan.machine_name)
    hs = engine.HostGradientStep(dp, *curve)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32).reshape(-1)).pin_memory()  # noqa: E731
    hu_h, presc_h, w_h = pin(c.grid.HU), pin(c.presc), pin(c.weights)
    dose_out = torch.empty(dp.n_vox, dtype=torch.float32).pin_memory()
    grad_out = torch.empty(dp.n_spots, dtype=torch.float32).pin_memory()
    obj_out = torch.empty(1, dtype=torch.float64).pin_memory()
    rng = np.random.default_rng(4)
    for _ in range(2):
        mu_h = pin(rng.uniform(0.5, 2.0, dp.n_spots))
        hs(hu_h, presc_h, w_h, mu_h, dose_out, grad_out, obj_out)
        torch.cuda.synchronize()
        dev = dp.device
        rlsp = engine.rlsp_from_hu(hu_h.to(dev), *curve)
        dp.compute_wet(rlsp)
        dose = dp.forward(dp.to_sorted(mu_h.to(dev)))
        resid = torch.empty_like(dose)
        obj = engine.objective(dose, presc_h.to(dev), w_h.to(dev), resid)
        grad = dp.to_plan(dp.adjoint(resid))
        assert torch.equal(dose_out, dose.cpu())
        g = grad.cpu()
        assert float((grad_out - g).abs().max()) <= 1e-5 * float(g.abs().max())
        assert float(obj_out[0]) == float(obj.item())
