"""The Energy Natural Gradient optimizer (fwi.py) on the CPU, against the
behaviour of sciml_solver/EnergyNaturalGradient.jl: the log-grid line
search (:155-177), the exact and probe Gram matrices (:63-112), the
regularised solve (:128-137), step! (:239-276) and optimize!'s stopping
rule (:294-321).  The seismic FWIProblem runs on the GPU
(test_gpu_fwi.py); here only its argument checks."""
import math

import numpy as np
import pytest

from viscoelasticinversion_b200 import fwi, media


def test_line_search_grid_first_minimum_and_batch():
    seen = []

    def loss(t):
        seen.append(float(t[0]))
        return (t[0] - 0.9) ** 2

    eta, best = fwi.line_search_log(loss, [1.0], [1.0], n_points=10, bounds=(1e-6, 1.0))
    grid = 10.0 ** np.linspace(-6.0, 0.0, 10)
    assert np.allclose(1.0 - np.array(seen), grid, rtol=1e-8, atol=0)  # 1 - (1 - η) cancels
    losses = (1.0 - grid - 0.9) ** 2
    assert eta == pytest.approx(grid[int(np.argmin(losses))]) and best == pytest.approx(losses.min())
    # one call for all trials gives the same answer
    eta_b, best_b = fwi.line_search_log(None, [1.0], [1.0], n_points=10, bounds=(1e-6, 1.0),
                                        batch_loss_fn=lambda ts: [loss(t) for t in ts])
    assert (eta_b, best_b) == (eta, best)
    # equal losses: the first (smallest) step wins
    eta_c, _ = fwi.line_search_log(lambda t: 3.0, [0.0], [1.0], n_points=5, bounds=(1e-3, 1.0))
    assert eta_c == pytest.approx(1e-3)


def test_exact_gram_step_solves_weighted_quadratic():
    w = np.array([1.0, 4.0, 0.25])
    target = np.array([0.3, -0.2, 1.5])
    loss = lambda t: 0.5 * float(np.sum(w * (t - target) ** 2))
    grad = lambda t: w * (t - target)
    # sensitivities sqrt(w_i) e_i: G = diag(w), natural gradient = t - target
    sens = lambda t: [math.sqrt(w[i]) * np.eye(3)[i] for i in range(3)]
    opt = fwi.EnergyNaturalGradientOptimizer(n_probes=0, regularization=1e-12)
    st = fwi.OptimizationState(np.zeros(3))
    l, eta = fwi.step(st, opt, loss, grad, sens)
    assert eta == pytest.approx(1.0) and l == pytest.approx(0.0, abs=1e-20)
    assert np.allclose(st.theta, target, rtol=0, atol=1e-10)
    assert st.iteration == 1 and st.loss_history == [l] and st.eta_history == [eta]


def test_gram_matrices_and_natural_gradient():
    s = [np.array([1.0, 2.0]), np.array([0.0, 3.0])]
    G = fwi.compute_gram_exact(s)
    assert np.array_equal(G, np.array([[5.0, 6.0], [6.0, 9.0]]))
    rho = np.array([2.0, 0.5])
    assert fwi.compute_gram_exact(s, rho)[0, 1] == pytest.approx(3.0)
    # identity JVP: <z, z> = p for Rademacher z, so the diagonal is exactly p
    Gs = fwi.compute_gram_stochastic(lambda z: z, 4, 7, rng=np.random.default_rng(1))
    assert np.allclose(np.diag(Gs), 4.0) and np.allclose(Gs, Gs.T)
    g = np.array([1.0, 1.0])
    assert np.allclose(fwi.compute_natural_gradient(G, g, 0.0), np.linalg.solve(G, g))


def test_identity_metric_and_stopping_rule():
    calls = []
    opt = fwi.EnergyNaturalGradientOptimizer(regularization=1.0, line_search_points=3,
                                             line_search_bounds=(0.25, 1.0))
    st = fwi.OptimizationState([2.0])
    # constant loss: every step changes it by 0, so optimize stops after the second
    out = fwi.optimize(st, opt, lambda t: 1.0, lambda t: np.array([4.0]), None, 50,
                       callback=lambda s, k, l, e: calls.append((k, l, e)))
    assert out is st and st.iteration == 2 and len(calls) == 2
    # identity metric: direction grad / (1 + reg) = 2, first grid step 0.25 (ties)
    assert np.allclose(st.theta, [2.0 - 2 * 0.25 * 2.0])


def test_fwi_problem_checks_its_arguments():
    w = media.homogeneous_iso(nx=64, nz=48, nt=10, pml=6, nrec=4)
    obs = [np.zeros((2, 4, 10))]
    with pytest.raises(ValueError, match="planes"):
        fwi.FWIProblem(w, [w], obs, planes=("c11",))
    with pytest.raises(ValueError, match="observed"):
        fwi.FWIProblem(w, [w, w], obs)
    other = media.homogeneous_iso(nx=72, nz=48, nt=10, pml=6, nrec=4)
    with pytest.raises(ValueError, match="grid"):
        fwi.FWIProblem(w, [other], obs)


def test_sensitivities_and_jvp_by_central_differences():
    A = np.array([[1.0, 2.0, 0.0], [0.5, -1.0, 3.0]])
    forward = lambda t: np.array([A @ t, np.sin(t).sum() * np.ones(2)])  # u: [2, 2]
    theta = np.array([0.3, -0.7, 1.1])
    sens = fwi.compute_sensitivities_forwardmode(forward, theta)
    for i in range(3):
        exact = np.array([A[:, i], np.cos(theta[i]) * np.ones(2)])
        assert np.allclose(sens[i], exact, rtol=1e-8, atol=1e-9)
    calls = []
    batched = fwi.compute_sensitivities_forwardmode(
        forward, theta, forward_batch=lambda ts: calls.append(len(ts)) or [forward(t) for t in ts])
    assert calls == [6] and all(np.array_equal(a, b) for a, b in zip(sens, batched))
    jvp = fwi.make_jvp_function(forward, theta)
    v = np.array([1.0, -2.0, 0.5])
    exact = np.array([A @ v, np.dot(np.cos(theta), v) * np.ones(2)])
    assert np.allclose(jvp(v), exact, rtol=1e-8, atol=1e-9)
    # with these, the optimizer's exact-Gram branch runs end to end
    G = fwi.compute_gram_exact(sens)
    assert np.allclose(G, G.T) and np.all(np.linalg.eigvalsh(G) > -1e-9)
    Gs = fwi.compute_gram_stochastic(jvp, 3, 5, rng=np.random.default_rng(0))
    assert Gs.shape == (3, 3) and np.allclose(Gs, Gs.T)
