"""Capped adjoint tapes (binomial checkpointing) against the fixed-interval
tape on the GPU.

The capped backward pass recomputes states from fewer checkpoints and tau
from the recomputed states; the forward arithmetic is deterministic, so the
gradient must equal the fixed-interval one (asserted to 1e-14 relative L2;
equal bit for bit is expected).  Caps from generous down to the minimum
exercise every schedule shape: no advances, binomial splits, and the
one-slot case where each chunk is reached from the first checkpoint."""
import numpy as np
import pytest

from exadglm_b200 import problem as P
from exadglm_b200.capi import DglmError, Solver

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


@pytest.mark.parametrize("phys,N,nsteps", [("euler", 4, 37), ("euler", 3, 24),
                                           ("advection", 3, 19)])
def test_capped_gradient_equals_fixed_interval(phys, N, nsteps):
    if phys == "euler":
        prob = P.euler_sine(n=3, N=N, noise=1e-3, seed=7)
    else:
        prob = P.advection_gaussian(n=3, N=N, width2=0.05)
    rng = np.random.default_rng(3)
    u0 = prob.u0.reshape(prob.nvar, -1)
    lamT = rng.standard_normal(u0.shape)
    s = Solver(prob)
    s.set_state(u0)
    s.adjoint_record(nsteps, 5)
    uT = s.get_state()
    ref = s.adjoint_backward(lamT)
    fixed_bytes = s.adjoint_tape_bytes()
    # the smallest accepted cap, found by halving from the fixed tape's size
    seen = set()
    for cap in (4 * fixed_bytes, fixed_bytes, fixed_bytes // 2, fixed_bytes // 4,
                fixed_bytes // 8):
        s.set_state(u0)
        try:
            s.adjoint_record_capped(nsteps, cap)
        except DglmError as e:
            assert "minimum tape" in str(e)
            continue
        assert s.adjoint_tape_bytes() <= cap
        assert rel(s.get_state(), uT) <= 1e-15        # the recording is the same run
        leaf, slots, adv = s.adjoint_tape_plan()
        g1 = s.adjoint_backward(lamT)
        g2 = s.adjoint_backward(lamT)                  # second pass: no prestored spine
        e1, e2 = rel(g1, ref), rel(g2, ref)
        print(f"{phys} N={N} cap {cap / 2**20:.1f} MiB: leaf {leaf} slots {slots} "
              f"advance steps {adv}: rel {e1:.1e} / {e2:.1e} "
              f"(bit-identical: {np.array_equal(g1, ref)})")
        assert e1 <= 1e-14 and e2 <= 1e-14, (e1, e2)
        seen.add((leaf, slots))
        with pytest.raises(DglmError, match="capped recording"):
            s.adjoint_replay()
    assert len(seen) >= 2, seen
    # below the minimum: refused with the minimum named
    s.set_state(u0)
    with pytest.raises(DglmError, match="minimum tape"):
        s.adjoint_record_capped(nsteps, 1 << 16)
    s.close()


def test_capped_tape_fits_config2_size():
    """Euler N=4 at 196,608 tets, 200 steps, the tape capped at 8 GiB (a
    fixed-interval tape every 50 steps would need about 60 GB): the backward
    pass runs and its gradient is finite and non-zero."""
    prob = P.euler_sine(n=32, N=4, cfl=0.4)
    s = Solver(prob)
    s.set_state(prob.u0)
    cap = 8 << 30
    s.adjoint_record_capped(200, cap)
    assert s.adjoint_tape_bytes() <= cap
    leaf, slots, adv = s.adjoint_tape_plan()
    lamT = np.zeros((prob.nvar, prob.K * prob.Np))
    lamT[0] = 1.0
    g = s.adjoint_backward(lamT)
    print(f"config-2 size: leaf {leaf} slots {slots} advance steps {adv}, "
          f"tape {s.adjoint_tape_bytes() / 2**30:.2f} GiB, |g| {np.linalg.norm(g):.3e}")
    assert np.all(np.isfinite(g)) and np.linalg.norm(g) > 0
    s.close()
