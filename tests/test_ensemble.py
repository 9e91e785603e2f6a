"""dglm_run_ensemble: independent initial states through one handle with the
host<->device copies overlapped with the compute.  Each member's result is
bit-identical to dglm_set_state + dglm_step + dglm_get_state on its own."""
import numpy as np
import pytest

from exadglm_b200 import problem as P

pytestmark = pytest.mark.gpu


def members(prob, count, seed=0):
    rng = np.random.default_rng(seed)
    u0 = np.asarray(prob.u0).reshape(prob.nvar, -1)
    return [u0 * (1 + 1e-3 * rng.standard_normal(u0.shape)) for _ in range(count)]


def sequential(s, states, nsteps):
    out = []
    for u in states:
        s.set_state(u)
        s.step(nsteps)
        out.append(s.get_state())
    return out


@pytest.mark.parametrize("phys", ["euler", "advection"])
def test_ensemble_matches_sequential(phys):
    from exadglm_b200.capi import Solver
    prob = (P.euler_sine(n=3, N=4, noise=1e-3, seed=2) if phys == "euler"
            else P.advection_gaussian(n=3, N=4, width2=0.05))
    states = members(prob, 5)
    s = Solver(prob)
    ref = sequential(s, states, 6)
    t_ref = s.time()
    got = s.run_ensemble(states, 6)
    for i, (a, b) in enumerate(zip(got, ref)):
        np.testing.assert_array_equal(a, b, err_msg=f"member {i}")
    assert s.time() == t_ref            # the handle holds the last member
    np.testing.assert_array_equal(s.get_state(), ref[-1])
    s.close()


def test_ensemble_pinned_overlap_and_reuse():
    """Page-locked buffers (the overlapped path), an odd member count, two
    calls on the same handle, and the handle still usable by dglm_step."""
    import torch
    from exadglm_b200.capi import Solver
    prob = P.euler_sine(n=4, N=3, noise=1e-3, seed=3)
    states = members(prob, 7, seed=1)
    s = Solver(prob)
    ref = sequential(s, states, 3)
    nv = prob.nvar
    hin = [torch.from_numpy(u).pin_memory() for u in states]
    hout = [torch.empty_like(x).pin_memory() for x in hin]
    for _ in range(2):
        for o in hout:
            o.fill_(float("nan"))
        bad = s.run_ensemble_ptrs([[x[v].data_ptr() for v in range(nv)] for x in hin],
                                  [[o[v].data_ptr() for v in range(nv)] for o in hout], 3)
        assert bad == -1
        for i in range(len(states)):
            np.testing.assert_array_equal(hout[i].numpy(), ref[i], err_msg=f"member {i}")
    # per member: finite check, wave speeds, then 9 kernels per Euler step
    # (begin, tau, five stages, wave speeds, end)
    assert s.kernel_launches() == len(states) * (2 + 9 * 3)
    s.step(2)
    s.sync()
    s.set_state(states[-1])
    s.step(5)
    np.testing.assert_array_equal(s.get_state(), sequential(s, [states[-1]], 5)[0])
    s.close()


def test_ensemble_reports_first_nonfinite_member():
    from exadglm_b200.capi import DglmError, Solver
    prob = P.euler_sine(n=3, N=3, noise=1e-3, seed=4)
    states = members(prob, 4, seed=2)
    states[2] = states[2].copy()
    states[2][0, 17] = np.nan
    s = Solver(prob)
    ref = sequential(s, [states[0], states[1], states[3]], 2)
    outs = [np.empty_like(u) for u in states]
    nv = prob.nvar
    with pytest.raises(DglmError):
        s.run_ensemble_ptrs([[u[v].ctypes.data for v in range(nv)] for u in states],
                            [[o[v].ctypes.data for v in range(nv)] for o in outs], 2)
    assert s.first_bad == 2
    for i, r in zip((0, 1, 3), ref):
        np.testing.assert_array_equal(outs[i], r)
    s.close()


def test_ensemble_on_a_fresh_handle():
    """The first call on a handle captures the step graph inside the
    pipelined loop (copies and event waits still queued on its stream)."""
    from exadglm_b200.capi import Solver
    prob = P.euler_sine(n=3, N=4, noise=1e-3, seed=7)
    states = members(prob, 3, seed=5)
    with Solver(prob) as fresh, Solver(prob) as ref_solver:
        got = fresh.run_ensemble(states, 4)
        ref = sequential(ref_solver, states, 4)
        for i, (a, b) in enumerate(zip(got, ref)):
            np.testing.assert_array_equal(a, b, err_msg=f"member {i}")
