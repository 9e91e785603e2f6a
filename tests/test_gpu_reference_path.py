"""The reference's own GPU path (dim3/src/cuda/euler_nopad_*.cu: its CUDA
kernels and cuBLAS batched DGEMMs, compiled here from its sources for sm_100a
by oracle/build_ref.py) against this library's FP64 path on the same mesh and
state: the two GPU implementations agree to the FP64 parity bar.  Skipped
where oracle/_ref holds no GPU build (the reference tree was absent when the
checker was built)."""
import numpy as np
import pytest

import oracle
from exadglm_b200 import problem as P
from exadglm_b200.capi import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not oracle.gpu_ref_available(4), reason="reference GPU build absent")
def test_reference_gpu_path_matches_fp64():
    prob = P.euler_sine(n=6, N=4, noise=1e-3, seed=11)      # CFL 0.4, gamma 1.4, tau 1.2
    ref = oracle.RefGpuSolver(prob)
    assert ref.run(10) == 10
    ur = ref.get_state()
    tr, dtr, nr = ref.time()
    ref.close()
    s = Solver(prob)
    s.step(10)
    s.sync()
    u = s.get_state()
    t, dt, n = s.time()
    s.close()
    err = float(np.linalg.norm(u - ur) / np.linalg.norm(ur))
    print(f"10 steps: rel L2 {err:.3e}, t {t!r} vs {tr!r}")
    assert n == nr == 10
    assert abs(t - tr) <= 1e-13 * tr and abs(dt - dtr) <= 1e-13 * dtr
    assert err < 1e-12
