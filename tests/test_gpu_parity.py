"""GPU parity: the CUDA path (libdglm.so through its C ABI) against the
oracle on the same seeded inputs.

Tolerances: the state after n LSERK steps agrees to 1e-12 relative L2 (the
FP64 bar of the hot path); one right-hand side to 1e-12 relative L2 of the
right-hand side (it carries cancellation, the oracle itself agrees with the
compiled reference to ~3e-14 there); time and dt to 1e-14 relative.
"""
import numpy as np
import pytest

import oracle
from exadglm_b200 import problem as P
from exadglm_b200.capi import Solver

pytestmark = pytest.mark.gpu

TOL_STATE = 1e-12
TOL_RHS = 1e-12
ORDERS = [1, 2, 3, 4, 5, 6, 7, 8]


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def make(phys, N, n=3):
    if phys == "advection":
        return P.advection_gaussian(n=n, N=N, width2=0.05)
    return P.euler_sine(n=n, N=N, noise=1e-3, seed=N)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    torch.cuda.init()
    return torch


@pytest.mark.parametrize("phys", ["advection", "euler"])
@pytest.mark.parametrize("N", ORDERS)
def test_rhs_matches_oracle(torch_cuda, phys, N):
    torch = torch_cuda
    prob = make(phys, N)
    s = Solver(prob)
    u = torch.tensor(prob.u0, device="cuda", dtype=torch.float64)
    r = torch.empty_like(u)
    s.rhs_device([u[v].data_ptr() for v in range(prob.nvar)],
                 [r[v].data_ptr() for v in range(prob.nvar)])
    ref = oracle.Oracle(prob).rhs()
    assert rel(r.cpu().numpy(), ref["utmp"]) < TOL_RHS
    s.close()


@pytest.mark.parametrize("phys", ["advection", "euler"])
@pytest.mark.parametrize("N", ORDERS)
def test_steps_match_oracle(phys, N):
    prob = make(phys, N)
    s = Solver(prob)
    s.step(10)
    s.sync()
    u = s.get_state()
    t, dt, ts = s.time()
    hist = s.dt_history(0, 10)
    uo, _, clk, ho = oracle.Oracle(prob).run(10)
    assert ts == 10
    assert abs(t - clk.t) <= 1e-14 * clk.t
    np.testing.assert_allclose(hist, ho, rtol=1e-14)
    assert rel(u, uo) < TOL_STATE
    s.close()


def test_tmax_clip_matches_oracle():
    """The last step is shortened to land on tmax; later steps change nothing
    (euler_time.cpp:54-57)."""
    prob = P.euler_sine(n=3, N=3, tmax=0.0123)
    s = Solver(prob)
    s.step(40)
    s.sync()
    t, dt, ts = s.time()
    uo, _, clk, ho = oracle.Oracle(prob).run(40)
    assert ts == clk.tstep and t == pytest.approx(0.0123, rel=0, abs=1e-15)
    np.testing.assert_allclose(s.dt_history(0, ts), ho, rtol=1e-14)
    assert rel(s.get_state(), uo) < TOL_STATE
    s.close()


def test_fixed_dt_matches_oracle():
    prob = P.euler_sine(n=3, N=4, noise=1e-3)
    s = Solver(prob)
    s.step(6, dt=1e-3)
    uo, _, clk, _ = oracle.Oracle(prob).run(6, dt_fixed=1e-3)
    assert rel(s.get_state(), uo) < TOL_STATE
    s.close()


def test_matrix_order_f_equals_c():
    """Operators given column-major (the GPU datain) give the same result."""
    prob = P.euler_sine(n=3, N=4, noise=1e-3)
    a = Solver(prob, matrix_order="c")
    b = Solver(prob, matrix_order="f")
    a.step(3)
    b.step(3)
    np.testing.assert_array_equal(a.get_state(), b.get_state())
    a.close()
    b.close()


def test_state_roundtrip_and_restart():
    """(u, t) restarts: k is reset at stage 0 because rka[0] = 0."""
    prob = P.euler_sine(n=3, N=3, noise=1e-3)
    s = Solver(prob)
    s.step(4)
    mid = s.get_state()
    s.step(4)
    end = s.get_state()
    s.set_state(mid)
    s.step(4)
    assert rel(s.get_state(), end) < 1e-14
    s.close()


@pytest.mark.parametrize("phys", ["advection", "euler"])
@pytest.mark.parametrize("N", ORDERS)
def test_every_variant_matches_oracle(phys, N):
    """Each compiled tile shape (SIMT and FP64 tensor-core DMMA engines) gives
    the oracle's answer."""
    from exadglm_b200.capi import variants
    prob = make(phys, N)
    uo, _, _, _ = oracle.Oracle(prob).run(3)
    for v, desc in variants(phys, N, "fp64"):
        s = Solver(prob)
        s.set_variant(v)
        s.step(3)
        assert rel(s.get_state(), uo) < TOL_STATE, (v, desc)
        s.close()
