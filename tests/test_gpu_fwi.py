"""One FWI iteration on the GPU (fwi.FWIProblem with the Energy Natural
Gradient optimizer): two ISO shots, the observed data from the FP64 oracle
on a true model whose λ and μ differ from the start model by a smooth 4 %
bump.  The batched loss (every trial model and shot in one vi_batch run)
agrees with the gradient path's misfit, and a step along the GPU gradient,
its length picked by the log-grid line search, lowers the misfit."""
import dataclasses

import numpy as np
import pytest

from viscoelasticinversion_b200 import fwi, media

pytestmark = pytest.mark.gpu

LOSS_RTOL = 1e-3  # FP32 traces against FP64 observations: J agrees to ~1e-4 between kernels


def _shot(src):
    return media.homogeneous_iso(nx=96, nz=80, nt=240, pml=12, nrec=16, src=src)


def test_fwi_step_lowers_the_misfit(oracle_lib):
    shots = [_shot((30, 30)), _shot((66, 30))]
    jj, ii = np.mgrid[0:80, 0:96]
    bump = np.exp(-((ii - 48) ** 2 + (jj - 22) ** 2) / (2 * 8.0**2))
    obs = []
    for w in shots:
        med = dict(w.medium)
        med["c13"] = med["c13"] * (1 + 0.04 * bump)
        med["c55"] = med["c55"] * (1 + 0.04 * bump)
        obs.append(oracle_lib.run(dataclasses.replace(w, medium=med), precision="f64")[0])
    prob = fwi.FWIProblem(shots[0], shots, obs, planes=("c13", "c55"), precision="f32")
    try:
        theta0 = np.zeros(prob.n_params)
        J0 = prob.loss(theta0)
        g0 = prob.grad(theta0)
        assert J0 > 0 and np.all(np.isfinite(g0)) and np.abs(g0).max() > 0
        (Jb,) = prob.batch_loss([theta0])
        assert abs(Jb - J0) <= LOSS_RTOL * J0, (Jb, J0)
        h = 0.05 / np.abs(g0).max()  # the longest trial moves a cell by 5 %
        opt = fwi.EnergyNaturalGradientOptimizer(line_search_points=6,
                                                 line_search_bounds=(1e-3 * h, h))
        st = fwi.OptimizationState(theta0)
        loss, eta = fwi.step(st, opt, prob.loss, prob.grad, None, prob.batch_loss)
        assert st.iteration == 1 and 1e-3 * h <= eta <= h * (1 + 1e-12)
        assert loss < J0, (loss, J0)
        assert abs(prob.loss(st.theta) - loss) <= LOSS_RTOL * loss
    finally:
        prob.close()
