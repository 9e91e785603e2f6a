"""The oracle's discrete adjoint (dglm_oracle.c: orc_rhs_adjoint, orc_adjoint)
against central finite differences of the oracle's own frozen-dt/tau run.
The reference has no adjoint; the forward it differentiates is the pinned
oracle step.  CPU only."""
import numpy as np
import pytest

import oracle
from exadglm_b200 import problem as P


def make(phys, N):
    if phys == "euler":
        return P.euler_sine(n=2, N=N, noise=1e-2, seed=N)
    return P.advection_gaussian(n=2, N=N, width2=0.05)


@pytest.mark.parametrize("phys", ["euler", "advection"])
@pytest.mark.parametrize("N", [1, 2, 3, 4])
def test_step_adjoint_matches_finite_differences(phys, N):
    prob = make(phys, N)
    O = oracle.Oracle(prob)
    rng = np.random.default_rng(100 + N)
    u0 = prob.u0.reshape(prob.nvar, -1)
    _, dt, tau = O.run_record(4, u0)
    lamT = rng.standard_normal(u0.shape)
    g = O.adjoint(u0, dt, tau, lamT)
    d = rng.standard_normal(u0.shape) * np.abs(u0).max()
    errs = []
    for h in (1e-4, 1e-5, 1e-6):
        up = O.run_frozen(u0 + h * d, dt, tau)
        um = O.run_frozen(u0 - h * d, dt, tau)
        fd = np.sum((up - um) * lamT) / (2 * h)
        errs.append(abs(fd - np.sum(g * d)) / abs(np.sum(g * d)))
    assert min(errs) < 1e-7, errs


@pytest.mark.parametrize("phys", ["euler", "advection"])
@pytest.mark.parametrize("N", [2, 4])
def test_rhs_adjoint_is_the_transpose(phys, N):
    """<(R(u + h d) - R(u - h d)) / 2h, mu> == <d, R'(u)^T mu> at frozen tau."""
    prob = make(phys, N)
    O = oracle.Oracle(prob)
    rng = np.random.default_rng(7 + N)
    u0 = prob.u0.reshape(prob.nvar, -1)
    tau = O.rhs(u0)["tau"]
    mu = rng.standard_normal(u0.shape)
    d = rng.standard_normal(u0.shape) * np.abs(u0).max()
    an = np.sum(O.rhs_adjoint(u0, tau, mu) * d)
    errs = []
    for h in (1e-4, 1e-5, 1e-6):
        fd = np.sum((O.rhs_frozen(u0 + h * d, tau) - O.rhs_frozen(u0 - h * d, tau)) * mu) / (2 * h)
        errs.append(abs(fd - an) / abs(an))
    assert min(errs) < 1e-7, errs
