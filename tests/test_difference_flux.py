"""The centred Euler volume flux in difference form, in FP32 (host check of
the algebra of the tensor-memory kernels' "vol=fp32-diff" variants,
vol_task_df in dglm_stage_tc.cuh and dglm_stage_tcb.cuh).

With the node-0 state (rho0, m0, E0) and du = u_i - u_0, both rounded to
FP32 once:
    dv_a = (dm_a - v0_a drho) / rho_i,   d(m_a v_b) = dm_a v0_b + m_a,i dv_b,
    dp = (gamma - 1) (dE - d(m.v) / 2),  d(H v_a) = dH v0_a + H_i dv_a,
no term cancels, so FP32 carries F(u_i) - F(u_0) to about 1e-7 of its size,
the precision of the TF32 split (2^-22) that follows it in the kernel.
Checked here against the same difference evaluated in FP64 on states like
the benchmark's (rho ~ 1 +- 0.2, v ~ (1, 0.5, 0.25), p ~ 1) with variations
from 1e-4 to 1e-1."""
import numpy as np

GAMMA = 1.4


def flux64(u):
    r, mx, my, mz, E = u
    vx, vy, vz = mx / r, my / r, mz / r
    p = (GAMMA - 1) * (E - 0.5 * (mx * vx + my * vy + mz * vz))
    H = E + p
    return np.array([[mx, mx * vx + p, my * vx, mz * vx, H * vx],
                     [my, mx * vy, my * vy + p, mz * vy, H * vy],
                     [mz, mx * vz, my * vz, mz * vz + p, H * vz]])


def dflux32(u0, du):
    """F(u0 + du) - F(u0) per direction, in the kernel's FP32 operation order."""
    f = np.float32
    r0, E0 = f(u0[0]), f(u0[4])
    m0 = [f(u0[1]), f(u0[2]), f(u0[3])]
    du = [f(x) for x in du]
    ir0 = f(1) / r0
    v0 = [m * ir0 for m in m0]
    H0 = E0 + f(GAMMA - 1) * (E0 - f(0.5) * (m0[0] * v0[0] + m0[1] * v0[1] + m0[2] * v0[2]))
    dr, dE = du[0], du[4]
    ir1 = f(1) / (r0 + dr)
    dv = [(du[1 + c] - v0[c] * dr) * ir1 for c in range(3)]
    m1 = [m0[c] + du[1 + c] for c in range(3)]
    dmv = [[du[1 + c] * v0[b] + m1[c] * dv[b] for b in range(3)] for c in range(3)]
    dp = f(GAMMA - 1) * (dE - f(0.5) * (dmv[0][0] + dmv[1][1] + dmv[2][2]))
    dH = dE + dp
    H1 = H0 + dH
    out = np.zeros((3, 5), dtype=np.float32)
    for b in range(3):
        out[b] = [du[1 + b], dmv[0][b], dmv[1][b], dmv[2][b], dH * v0[b] + H1 * dv[b]]
        out[b, 1 + b] += dp
    return out


def test_difference_form_matches_fp64_difference():
    rng = np.random.default_rng(11)
    errs = []
    for _ in range(4000):
        r = 1 + 0.2 * np.sin(rng.uniform(0, 2 * np.pi))
        v = np.array([1.0, 0.5, 0.25]) + 0.05 * rng.standard_normal(3)
        p = 1 + 0.05 * rng.standard_normal()
        u0 = np.array([r, r * v[0], r * v[1], r * v[2], p / (GAMMA - 1) + 0.5 * r * v @ v])
        du = u0 * 10 ** rng.uniform(-4, -1) * rng.standard_normal(5)
        ref = flux64(u0 + du) - flux64(u0)
        got = dflux32(u0, du).astype(np.float64)
        errs.extend(np.max(np.abs(got - ref), axis=1) / np.max(np.abs(ref), axis=1))
    errs = np.array(errs)
    print(f"relative error of dF: median {np.median(errs):.2e}, "
          f"99th percentile {np.quantile(errs, 0.99):.2e}, max {errs.max():.2e}")
    # about the split's own precision (2^-22 = 2.4e-7) for the bulk of states
    assert np.median(errs) < 2.4e-7
    assert np.quantile(errs, 0.99) < 2e-6


def test_constant_state_gives_zero():
    u0 = np.array([1.1, 1.1, 0.55, 0.275, 3.2])
    assert np.all(dflux32(u0, np.zeros(5)) == 0)
