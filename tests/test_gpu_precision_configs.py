"""Mixed precision at the full sizes of the Euler workloads, 200 steps each,
relative L2 of the whole state against the FP64 path from the same initial
state (the precision pattern's bar: <= 1e-6 after 200 steps).

* Euler N=4 on 32^3 x 6 = 196,608 tets, CFL 0.4: TF32x3 (the handle's
  default variant and every tensor-memory variant) <= 5e-7.
* Euler N=6 on 48^3 x 6 = 663,552 tets, CFL 0.4: TF32x3, BF16x6 and BF16x3
  (default variants, and the BF16 tensor-memory kernel) <= 1e-6.

The split operands are centred on each element's node-0 flux, which leaves
the right-hand side unchanged and shrinks the values the tensor cores see."""
import numpy as np
import pytest

from exadglm_b200 import problem as P
from exadglm_b200.capi import Solver, variants

pytestmark = pytest.mark.gpu

STEPS = 200


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def run(prob, precision, variant=None):
    s = Solver(prob, precision=precision, variant=variant)
    desc = variants("euler", prob.N)[s.variant()]
    s.step(STEPS)
    s.sync()
    u = s.get_state()
    s.close()
    return u, desc


def test_euler_n4_196608_tets():
    prob = P.euler_sine(n=32, N=4, cfl=0.4)
    ref, _ = run(prob, "fp64")
    cases = [None] + [v for v, d in variants("euler", 4, "tf32x3") if d.startswith("tc-")]
    for v in cases:
        u, desc = run(prob, "tf32x3", v)
        err = rel(u, ref)
        print(f"N=4 K={prob.K} tf32x3 {desc}: {STEPS}-step rel L2 {err:.3e}")
        assert err <= 5e-7, (desc, err)


def test_euler_n6_663552_tets():
    prob = P.euler_sine(n=48, N=6, cfl=0.4)
    ref, _ = run(prob, "fp64")
    cases = [("tf32x3", None), ("bf16x6", None), ("bf16x3", None)] + \
        [("bf16x3", v) for v, d in variants("euler", 6, "bf16x3") if d.startswith("tc-")]
    for prec, var in cases:
        u, desc = run(prob, prec, var)
        err = rel(u, ref)
        per_field = [rel(u[v], ref[v]) for v in range(prob.nvar)]
        print(f"N=6 K={prob.K} {prec} {desc}: {STEPS}-step rel L2 {err:.3e}, per field "
              + " ".join(f"{e:.2e}" for e in per_field))
        assert err <= 1e-6, (prec, desc, err)
