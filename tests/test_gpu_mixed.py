"""Mixed-precision contractions on the tcgen05 tensor cores (3-pass TF32 and
split BF16 with FP32 accumulation; state, fluxes and update in FP64) against
the FP64 oracle.  The mixed modes are not bit-compatible by design: each
test states its error bound.

A contraction's error is bounded against the size of its terms, not of its
result (the right-hand side is a sum of large terms that nearly cancel):
  s_i = sum_k |A_ik| |B_k|   over the volume and lift terms of output i,
  max_i |rhs_mixed,i - rhs_fp64,i| / s_i  <=  2^-20 (TF32x3), 2^-16 (BF16x3),
                                           2^-21 (BF16x6).
TF32x3 keeps ~22 significant bits per operand (measured ~2^-23), BF16x3 ~16
bits (measured ~2^-18), BF16x6 24 bits with six part products; every mode
sums its products in FP32 over 8 slices of K (tensor-memory accumulators
for tcgen05, register accumulators folded into FP64 for mma.sync).  The state after 20
steps is checked in relative L2 (TF32x3 and BF16x6 <= 1e-6, BF16x3 <= 1e-4).
"""
import numpy as np
import pytest

import oracle
from exadglm_b200 import problem as P
from exadglm_b200.capi import Solver, variants

pytestmark = pytest.mark.gpu

SCALED_TOL = {"tf32x3": 2.0 ** -20, "bf16x3": 2.0 ** -16, "bf16x6": 2.0 ** -21}
STATE_TOL = {"tf32x3": 1e-6, "bf16x3": 1e-4, "bf16x6": 1e-6}
# tcgen05 variants (Euler N=4, advection N=3) and split-precision mma.sync
# variants (orders whose tcgen05 operand images exceed shared memory)
CASES = [("euler", 4), ("advection", 3), ("euler", 5), ("euler", 6), ("advection", 6)]


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def make(phys, N):
    if phys == "advection":
        return P.advection_gaussian(n=3, N=N, width2=0.05)
    return P.euler_sine(n=3, N=N, noise=1e-3, seed=N)


def term_scale(prob, out):
    """s_i = sum_k |A_ik||B_k| per output node, from the oracle's fluxes."""
    re = prob.mesh.ref
    K, Np, NF, nv = prob.K, prob.Np, 4 * prob.Nfp, prob.nvar
    fR, fS, fT = (np.abs(out[k]).reshape(nv, K, Np) for k in ("fluxR", "fluxS", "fluxT"))
    fL = np.abs(out["fluxLM"]).reshape(nv, K, NF)
    s = (np.einsum("ij,vej->vei", np.abs(re.WDr), fR) + np.einsum("ij,vej->vei", np.abs(re.WDs), fS)
         + np.einsum("ij,vej->vei", np.abs(re.WDt), fT) + np.einsum("ij,vej->vei", np.abs(re.LIFT), fL))
    return s.reshape(nv, K * Np)


@pytest.mark.parametrize("prec", ["tf32x3", "bf16x3", "bf16x6"])
@pytest.mark.parametrize("phys,N", CASES)
def test_mixed_rhs_error(phys, N, prec):
    import torch
    prob = make(phys, N)
    out = oracle.Oracle(prob).rhs()
    ref = out["utmp"].reshape(prob.nvar, -1)
    scale = term_scale(prob, out)
    for v, desc in variants(phys, N, prec):
        s = Solver(prob, precision=prec, variant=v)
        u = torch.tensor(prob.u0, device="cuda", dtype=torch.float64)
        r = torch.empty_like(u)
        s.rhs_device([u[i].data_ptr() for i in range(prob.nvar)],
                     [r[i].data_ptr() for i in range(prob.nvar)])
        got = r.cpu().numpy()
        scaled = float(np.max(np.abs(got - ref) / scale))
        print(f"{desc}: max |d|/s = {scaled:.3e} (2^{np.log2(scaled):.1f}), rel L2 {rel(got, ref):.3e}")
        assert scaled < SCALED_TOL[prec], (desc, scaled)
        s.close()


@pytest.mark.parametrize("prec", ["tf32x3", "bf16x3", "bf16x6"])
@pytest.mark.parametrize("phys,N", CASES)
def test_mixed_steps_error(phys, N, prec):
    prob = make(phys, N)
    uo, _, _, _ = oracle.Oracle(prob).run(20)
    s = Solver(prob, precision=prec, variant=-1)
    s.step(20)
    s.sync()
    err = rel(s.get_state(), uo)
    print(f"{phys} N={N} {prec}: 20 steps rel L2 {err:.3e}")
    assert err < STATE_TOL[prec], err
    s.close()


@pytest.mark.parametrize("prec", ["tf32x3", "bf16x3", "bf16x6"])
@pytest.mark.parametrize("phys,N", CASES)
def test_every_mixed_variant_steps(phys, N, prec):
    """Every tile shape of the mode through full steps (the LSERK epilogue
    included, whether it reads the RK register from shared or global memory)."""
    prob = make(phys, N)
    uo, _, _, _ = oracle.Oracle(prob).run(5)
    for v, desc in variants(phys, N, prec):
        s = Solver(prob, precision=prec, variant=v)
        s.step(5)
        s.sync()
        err = rel(s.get_state(), uo)
        print(f"{desc}: 5 steps rel L2 {err:.3e}")
        assert err < STATE_TOL[prec], (desc, err)
        s.close()


def test_variant_of_other_precision_is_rejected():
    from exadglm_b200.capi import DglmError
    prob = make("euler", 4)
    s = Solver(prob, precision="tf32x3", variant=-1)
    fp64 = variants("euler", 4, "fp64")[0][0]
    with pytest.raises(DglmError):
        s.set_variant(fp64)
    s.close()
