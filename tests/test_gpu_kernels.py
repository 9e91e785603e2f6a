"""The per-kernel entry points (the reference's kernel split: calc_maxv,
calc_dt, update_tau, update_ub, calc_fluxLM, calc_fluxes, update_rhs,
lserk_stage) through the C ABI on caller-owned device arrays, each against
the oracle's output of the same step on the same state.  Tolerance 1e-13
relative (max norm over the array) per kernel; update_rhs, whose result is a
small difference of large terms, 1e-12 relative L2 (as the fused path's
rhs), in both matrix orders."""
import ctypes as C

import numpy as np
import pytest

import oracle
from exadglm_b200 import capi
from exadglm_b200 import problem as P

pytestmark = pytest.mark.gpu
TOL = 1e-13


def rel2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def relmax(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def make(phys, N):
    if phys == "euler":
        return P.euler_sine(n=3, N=N, noise=1e-3, seed=N)
    return P.advection_gaussian(n=3, N=N, width2=0.05)


@pytest.mark.parametrize("phys", ["euler", "advection"])
@pytest.mark.parametrize("N", [2, 4])
def test_per_kernel_entry_points_match_oracle(phys, N):
    import torch
    L = capi.lib()
    prob = make(phys, N)
    arr = prob.datain_arrays()
    ref = oracle.Oracle(prob).rhs()
    dev = torch.device("cuda")
    K, Np, NFF, nv = prob.K, prob.Np, 4 * prob.Nfp, prob.nvar
    ph = capi.EULER if phys == "euler" else capi.ADVECTION

    def d64(a):
        return torch.tensor(np.ascontiguousarray(np.asarray(a, np.float64).ravel()), device=dev)

    def d32(a):
        return torch.tensor(np.ascontiguousarray(np.asarray(a, np.int32).ravel()), device=dev)

    def P_(t):
        return C.c_void_p(t.data_ptr())

    def table(ts):
        return capi.ptr_table([t.data_ptr() for t in ts])

    Fmask, vmapP, vmapF = d32(arr["Fmask"]), d32(arr["vmapP"]), d32(arr["vmapF"])
    Fscale, nx, ny, nz = (d64(arr[k]) for k in ("Fscale", "nx", "ny", "nz"))
    geo = [d64(arr[k]) for k in ("rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz")]
    u = d64(prob.u0).reshape(nv, K * Np)
    us = [u[v] for v in range(nv)]
    if phys == "euler":
        vx = vy = vz = None
        vel = (None, None, None)
    else:
        vx, vy, vz = (d64(prob.vel[q]) for q in range(3))
        vel = (P_(vx), P_(vy), P_(vz))
    maxv = torch.empty(4 * K, dtype=torch.float64, device=dev)
    maxv_fs = torch.empty_like(maxv)
    capi.check(L.dglm_calc_maxv(ph, N, K, prob.gamma, P_(Fmask), P_(Fscale),
                                table(us) if phys == "euler" else None, *vel, P_(maxv),
                                P_(maxv_fs), None))
    dt = torch.empty(1, dtype=torch.float64, device=dev)
    capi.check(L.dglm_calc_dt(N, K, prob.cfl, P_(maxv_fs), P_(dt), None))
    tau = torch.empty_like(maxv)
    capi.check(L.dglm_update_tau(K, prob.tau_scale, P_(vmapF), P_(maxv), P_(tau), None))
    ub = torch.empty((nv, K * NFF), dtype=torch.float64, device=dev)
    capi.check(L.dglm_update_ub(N, nv, K, P_(Fmask), P_(vmapP), table(us),
                                table([ub[v] for v in range(nv)]), None))
    fLM = torch.empty_like(ub)
    capi.check(L.dglm_calc_fluxLM(ph, N, K, prob.gamma, P_(Fmask), P_(nx), P_(ny), P_(nz),
                                  P_(tau), P_(Fscale), *vel, table([ub[v] for v in range(nv)]),
                                  table(us), table([fLM[v] for v in range(nv)]), None))
    fR, fS, fT = (torch.empty_like(u) for _ in range(3))
    capi.check(L.dglm_calc_fluxes(ph, N, K, prob.gamma, table(geo), *vel, table(us),
                                  table([fR[v] for v in range(nv)]),
                                  table([fS[v] for v in range(nv)]),
                                  table([fT[v] for v in range(nv)]), None))
    outs = {}
    for order in ("c", "f"):
        ops = [d64(np.asarray(arr[k]).ravel(order="F" if order == "f" else "C"))
               for k in ("WDr", "WDs", "WDt", "LIFT")]
        utmp = torch.empty_like(u)
        capi.check(L.dglm_update_rhs(N, nv, K, *(P_(o) for o in ops), order.encode(),
                                     table([fR[v] for v in range(nv)]),
                                     table([fS[v] for v in range(nv)]),
                                     table([fT[v] for v in range(nv)]),
                                     table([fLM[v] for v in range(nv)]),
                                     table([utmp[v] for v in range(nv)]), None))
        outs[order] = utmp
    torch.cuda.synchronize()
    got = {"maxv": maxv, "tau": tau, "ub": ub, "fluxLM": fLM, "fluxR": fR, "fluxS": fS,
           "fluxT": fT, "utmp": outs["c"]}
    for k, t in got.items():
        e = (rel2 if k == "utmp" else relmax)(t.cpu().numpy(), ref[k])
        print(f"{phys} N={N} {k}: {e:.2e}")
        assert e <= (1e-12 if k == "utmp" else TOL), (k, e)
    assert rel2(outs["f"].cpu().numpy(), ref["utmp"]) <= 1e-12
    assert abs(dt.item() - ref["dt"]) <= TOL * ref["dt"]

    # lserk_stage: k = a k + dt utmp, u = u + b k
    a, b_, dts = -0.4, 0.3, 1.7e-3
    k0 = torch.randn_like(u)
    k1, u1 = k0.clone(), u.clone()
    capi.check(L.dglm_lserk_stage(N, nv, K, dts, a, b_, table([outs["c"][v] for v in range(nv)]),
                                  table([k1[v] for v in range(nv)]),
                                  table([u1[v] for v in range(nv)]), None))
    torch.cuda.synchronize()
    kr = a * k0.cpu().numpy() + dts * outs["c"].cpu().numpy()
    assert relmax(k1.cpu().numpy(), kr) <= TOL
    assert relmax(u1.cpu().numpy(), u.cpu().numpy() + b_ * kr) <= TOL
