"""Batched advection (dglm_batch_*): many meshes of different size and order
advanced by one launch per stage, each instance against the single-mesh
solver and the oracle.

Tolerances: per instance, relative L2 against the single-mesh FP64 solver
<= 1e-13 and against the oracle <= 1e-12 (FP64, different summation order
in the contraction); per-instance dt and time equal the single solver's."""
import ctypes as C

import numpy as np
import pytest

import oracle
from exadglm_b200 import capi
from exadglm_b200 import problem as P


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def test_batch_rejects_euler_and_bad_arguments():
    L = capi.lib()
    d = capi.BatchDesc(physics=capi.EULER, cfl=0.5, tau_scale=1.2, tmax=1.0, device=0)
    h = C.c_void_p()
    assert L.dglm_batch_create(C.byref(d), C.byref(h)) == capi.ERR_UNSUPPORTED
    d.physics, d.cfl = capi.ADVECTION, -1.0
    assert L.dglm_batch_create(C.byref(d), C.byref(h)) == capi.ERR_INVALID
    assert L.dglm_batch_create(None, C.byref(h)) == capi.ERR_INVALID


def test_batch_instances_are_seeded_and_in_range():
    a = P.batch_instances(count=6, seed=11, n_range=(2, 3))
    b = P.batch_instances(count=6, seed=11, n_range=(2, 3))
    for p, q in zip(a, b):
        assert p.N == q.N and p.K == q.K and np.array_equal(p.u0, q.u0)
        assert 2 <= p.N <= 6 and p.K in (6 * 8, 6 * 27)
        v = np.asarray(p.vel)
        assert np.all(np.abs(v) <= 1) and np.all(v == v[:, :1])


@pytest.mark.gpu
def test_batch_matches_single_solver_and_oracle():
    probs = P.batch_instances(count=12, seed=3, n_range=(2, 4), orders=(2, 6))
    assert len({p.N for p in probs}) >= 3
    b = capi.BatchSolver(probs)
    nsteps = 6
    b.step(nsteps)
    b.sync()
    for i, p in enumerate(probs):
        got = b.get_state(i)
        s = capi.Solver(p, variant=-1)
        s.step(nsteps)
        s.sync()
        ref = s.get_state().ravel()
        t1, dt1, n1 = s.time()
        t2, dt2, n2 = b.time(i)
        s.close()
        uo, _, clk, _ = oracle.Oracle(p).run(nsteps)
        e1, e2 = rel(got, ref), rel(got, uo)
        print(f"instance {i} N={p.N} K={p.K}: vs single {e1:.2e}, vs oracle {e2:.2e}")
        assert e1 <= 1e-13 and e2 <= 1e-12, (i, e1, e2)
        assert n1 == n2 == nsteps and t1 == t2 and dt1 == dt2, (i, t1, t2, dt1, dt2)
    b.close()


@pytest.mark.gpu
def test_batch_clips_each_instance_to_tmax():
    probs = P.batch_instances(count=5, seed=4, n_range=(2, 3), orders=(2, 4), tmax=0.02)
    b = capi.BatchSolver(probs)
    b.step(40)
    b.sync()
    for i, p in enumerate(probs):
        s = capi.Solver(p, variant=-1)
        s.step(40)
        s.sync()
        assert rel(b.get_state(i), s.get_state().ravel()) <= 1e-13
        t1, _, n1 = s.time()
        t2, _, n2 = b.time(i)
        assert t2 == pytest.approx(0.02, abs=1e-15) and t1 == t2 and n1 == n2
        s.close()
    b.close()


@pytest.mark.gpu
def test_batch_config4_instances_match_single_solvers():
    """The first 16 instances of the 256-instance ensemble workload (seed 0:
    n in 4..24, N in 2..6, the full size distribution) batched, against one
    single-mesh solver per instance, 10 steps."""
    probs = P.batch_instances(count=16, seed=0)
    assert max(p.K for p in probs) > 6 * 12 ** 3 and len({p.N for p in probs}) >= 4
    b = capi.BatchSolver(probs)
    nsteps = 10
    b.step(nsteps)
    b.sync()
    worst = 0.0
    for i, p in enumerate(probs):
        s = capi.Solver(p)
        s.step(nsteps)
        s.sync()
        e = rel(b.get_state(i), s.get_state().ravel())
        t1, dt1, n1 = s.time()
        t2, dt2, n2 = b.time(i)
        s.close()
        worst = max(worst, e)
        assert e <= 1e-13, (i, p.N, p.K, e)
        assert n1 == n2 == nsteps and t1 == t2 and dt1 == dt2, (i, t1, t2)
    print(f"16 config-4 instances (K {min(p.K for p in probs)}..{max(p.K for p in probs)}): "
          f"worst rel L2 vs single solvers {worst:.2e}")
    b.close()
