"""dglm_calc_maxv_dt_static (scratch in a file-scope device array, no
allocation) against the existing pair dglm_calc_maxv + dglm_calc_dt on the
same device fields, through the C ABI, on two calls in a row.

Both compute maxv with the same arithmetic (one shared device function) and
dt from the same max (a max is independent of reduction order), so maxv and
dt must agree exactly; the tolerance is 0.  The calls after the first must
not change the device's free memory (nothing is allocated), and a call on a
second stream, ordered after the first, gives the same result (the scratch
is shared by every call; serialised calls do not interfere).  The size limit
is rejected on the host before any device call, so that check runs without a
GPU."""
import ctypes as C

import numpy as np
import pytest

from exadglm_b200 import capi
from exadglm_b200 import problem as P

MAX_ELEMENTS = 4194304


def _ptrs(ts):
    return capi.ptr_table([t.data_ptr() for t in ts])


def test_rejects_meshes_above_the_scratch_limit():
    L = capi.lib()
    one = (C.c_void_p * 5)(*([C.c_void_p(8)] * 5))
    st = L.dglm_calc_maxv_dt_static(1, 4, MAX_ELEMENTS + 1, 1.4, 0.4, C.c_void_p(8),
                                    C.c_void_p(8), one, None, None, None, C.c_void_p(8),
                                    C.c_void_p(8), None)
    assert st == capi.ERR_INVALID
    assert b"static scratch limit" in L.dglm_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("phys,N,n", [("euler", 4, 3), ("euler", 3, 8), ("advection", 3, 8)])
def test_matches_calc_maxv_plus_calc_dt_twice(phys, N, n):
    import torch
    L = capi.lib()
    prob = (P.euler_sine(n=n, N=N, noise=1e-3, seed=N) if phys == "euler"
            else P.advection_gaussian(n=n, N=N, width2=0.05))
    arr = prob.datain_arrays()
    dev = torch.device("cuda")
    K = prob.K
    Fmask = torch.tensor(np.asarray(arr["Fmask"], dtype=np.int32), device=dev)
    Fscale = torch.tensor(np.asarray(arr["Fscale"], dtype=np.float64).ravel(), device=dev)
    u = torch.tensor(np.asarray(prob.u0, dtype=np.float64).reshape(prob.nvar, -1), device=dev)
    us = [u[v] for v in range(prob.nvar)]
    if phys == "euler":
        u_tab, vel = _ptrs(us), (None, None, None)
        ph = capi.EULER
    else:
        vt = torch.tensor(np.asarray(prob.vel, dtype=np.float64), device=dev)
        u_tab, vel = None, tuple(C.c_void_p(vt[q].data_ptr()) for q in range(3))
        ph = capi.ADVECTION
    gamma, cfl = prob.gamma, prob.cfl

    maxv_ref = torch.empty(4 * K, dtype=torch.float64, device=dev)
    maxv_fs = torch.empty(4 * K, dtype=torch.float64, device=dev)
    dt_ref = torch.empty(1, dtype=torch.float64, device=dev)
    capi.check(L.dglm_calc_maxv(ph, N, K, gamma, C.c_void_p(Fmask.data_ptr()),
                                C.c_void_p(Fscale.data_ptr()), u_tab, *vel,
                                C.c_void_p(maxv_ref.data_ptr()), C.c_void_p(maxv_fs.data_ptr()),
                                None))
    capi.check(L.dglm_calc_dt(N, K, cfl, C.c_void_p(maxv_fs.data_ptr()),
                              C.c_void_p(dt_ref.data_ptr()), None))
    torch.cuda.synchronize()

    maxv = torch.empty(4 * K, dtype=torch.float64, device=dev)
    dt = torch.empty(1, dtype=torch.float64, device=dev)
    side = torch.cuda.Stream()

    def call_static(stream):
        maxv.fill_(-1.0)
        dt.fill_(-1.0)
        torch.cuda.synchronize()
        capi.check(L.dglm_calc_maxv_dt_static(ph, N, K, gamma, cfl,
                                              C.c_void_p(Fmask.data_ptr()),
                                              C.c_void_p(Fscale.data_ptr()), u_tab, *vel,
                                              C.c_void_p(maxv.data_ptr()),
                                              C.c_void_p(dt.data_ptr()),
                                              None if stream is None else
                                              C.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize()

    free_before = None
    for call in range(3):
        call_static(side if call == 2 else None)
        if call == 0:
            free_before = torch.cuda.mem_get_info()[0]
        assert torch.equal(maxv, maxv_ref), (phys, N, call)
        assert float(dt.item()) == float(dt_ref.item()), (call, dt.item(), dt_ref.item())
        assert float(dt.item()) > 0
    # the calls after the first allocated nothing on the device
    assert torch.cuda.mem_get_info()[0] == free_before
