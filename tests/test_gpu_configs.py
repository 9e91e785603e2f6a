"""The workloads at their own sizes.

* Advection, K = 3,072, N = 3 (Gaussian of width^2 0.01, v = (1, 0.5, 0.25),
  CFL 0.5): the full 100-step run against the oracle.
* Euler, K = 196,608, N = 4 (the benchmark workload): two steps against the
  oracle, then 200 steps checked by conservation.
* Euler, K = 663,552, N = 6: 20 steps checked by conservation.

Conservation is the size-independent property of this scheme: on a periodic
mesh the weak-form volume terms integrate to zero (Dr 1 = 0) and the trace
flux of a face cancels against its neighbour's (same average state, opposite
normal, symmetric tau), so the mass-weighted integral of every conserved
variable, sum_k J_k w^T u_k with w = M 1, changes only by rounding.  Bound:
the drift over the run is below 1e-12 of sum_k J_k |w|^T |u_k|.
"""
import numpy as np
import pytest

import oracle
from exadglm_b200 import problem as P
from exadglm_b200.capi import Solver

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def integrals(prob, u):
    """(integral of each variable, integral of its magnitude)."""
    m = prob.mesh
    w = m.ref.M.sum(axis=0)
    U = np.asarray(u).reshape(prob.nvar, prob.K, prob.Np)
    return (np.einsum("k,vki,i->v", m.J, U, w),
            np.einsum("k,vki,i->v", np.abs(m.J), np.abs(U), np.abs(w)))


def test_advection_K3072_N3_100_steps_against_oracle():
    prob = P.advection_gaussian()          # n = 8: K = 3,072, N = 3
    assert prob.K == 3072 and prob.N == 3
    uo, _, clk, dts = oracle.Oracle(prob).run(100)
    t_o = clk.t
    s = Solver(prob)
    s.step(100)
    s.sync()
    err = rel(s.get_state(), uo)
    t, _, ts = s.time()
    print(f"advection K=3072 N=3, 100 steps: rel L2 {err:.3e}")
    assert err < 1e-12 and ts == 100
    assert abs(t - t_o) <= 1e-14 * t_o
    np.testing.assert_allclose(s.dt_history(0, 100), dts, rtol=1e-14)
    s.close()


@pytest.fixture(scope="module")
def euler_n4_full():
    return P.euler_sine(n=32, N=4)          # K = 196,608


def test_euler_K196608_N4_two_steps_against_oracle(euler_n4_full):
    prob = euler_n4_full
    assert prob.K == 196608
    uo, _, _, _ = oracle.Oracle(prob).run(2)
    s = Solver(prob)
    s.step(2)
    s.sync()
    err = rel(s.get_state(), uo)
    print(f"euler K=196608 N=4, 2 steps: rel L2 {err:.3e}")
    assert err < 1e-12
    s.close()


@pytest.mark.parametrize("n,N,steps", [(32, 4, 200), (48, 6, 20)])
def test_euler_conservation_full_size(euler_n4_full, n, N, steps):
    prob = euler_n4_full if (n, N) == (32, 4) else P.euler_sine(n=n, N=N)
    s = Solver(prob)
    i0, mag = integrals(prob, prob.u0)
    s.step(steps)
    s.sync()
    i1, _ = integrals(prob, s.get_state())
    drift = np.abs(i1 - i0) / mag
    print(f"euler K={prob.K} N={N}, {steps} steps: drift / magnitude {drift}")
    assert s.time()[2] == steps
    assert np.all(drift < 1e-12), drift
    s.close()
