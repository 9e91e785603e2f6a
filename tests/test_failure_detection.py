"""Failure detection, injected on the host: corrupted input files and mesh
arrays are rejected with a status before any kernel runs, and the bounded
waits of the pipelined stage kernels report their expiry instead of hanging.

The expiry test shortens the bound of the kernels' hand-off waits to one
clock cycle (dglm_set_wait_limit), so the first wait for a tile's copies runs
out on every SM; each CTA then sets the error flag, waits with the normal
bound for its own copies and MMAs in flight, and leaves.  dglm_sync must
report it, and the handle (after a new state) and a fresh handle must step
as before.  Nothing here faults or traps a GPU."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from exadglm_b200 import build as _build
from exadglm_b200 import capi
from exadglm_b200 import problem as P
from test_launcher import notebook_launcher


def test_driver_rejects_truncated_datain(tmp_path):
    """A vmapP.bin shorter than K * 4 * Nfp stops dglm_main before it
    creates a handle (no GPU call)."""
    if not os.path.exists(_build.MAIN):
        pytest.skip("dglm_main not built")
    dg, _ = notebook_launcher(tmp_path, 5, nx=4, N=3, tmax=0.5)
    path = os.path.join(dg.datain_dir, "vmapP.bin")
    data = np.fromfile(path, dtype=np.int32)
    data[: data.size - 7].tofile(path)
    r = subprocess.run([_build.MAIN, "--datain", dg.datain_dir, "--dataout", str(tmp_path),
                        "--physics", "euler", "--tmax", "0.5", "--matrix-order", "f"],
                       stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    assert r.returncode == 1, r.stderr
    assert "vmapP.bin holds" in r.stderr and "expected" in r.stderr, r.stderr


def _prob():
    return P.euler_sine(n=3, N=4, noise=1e-3, seed=3)


def _upload(prob, arr):
    """dglm_create + dglm_upload_mesh with the given datain arrays; returns
    (status, last error)."""
    L = capi.lib()
    d = capi.Desc()
    d.N, d.K, d.physics, d.precision = prob.N, prob.K, capi.EULER, capi.PREC_FP64
    d.cfl, d.gamma, d.tau_scale, d.tmax, d.device = prob.cfl, prob.gamma, prob.tau_scale, \
        prob.tmax, 0
    h = capi._P()
    capi.check(L.dglm_create(d, h))
    m, keep = capi.mesh_arrays(prob, arr)
    st = L.dglm_upload_mesh(h, m)
    msg = L.dglm_last_error().decode()
    L.dglm_destroy(h)
    return st, msg


@pytest.mark.gpu
@pytest.mark.parametrize("name,index,value,msg", [
    ("vmapP", 17, "K*Np", "vmapP entry outside"),
    ("vmapP", 0, -1, "vmapP entry outside"),
    ("vmapF", 5, "4K", "vmapF entry outside"),
    ("Fmask", 3, "Np", "Fmask entry outside"),
    ("rx", 11, np.nan, "non-finite metric"),
    ("Fscale", 2, np.inf, "non-finite face array"),
    ("WDr", 4, np.nan, "non-finite operator entry"),
])
def test_upload_rejects_corrupted_mesh(name, index, value, msg):
    prob = _prob()
    arr = {k: np.array(v, copy=True) for k, v in prob.datain_arrays().items()}
    if isinstance(value, str):
        value = {"K*Np": prob.K * prob.Np, "4K": 4 * prob.K, "Np": prob.Np}[value]
    flat = arr[name].reshape(-1)
    flat[index] = value
    st, err = _upload(prob, arr)
    assert st == capi.ERR_INVALID, (st, err)
    assert msg in err, err


@pytest.mark.gpu
def test_set_state_rejects_nonfinite_values():
    prob = _prob()
    s = capi.Solver(prob)
    u = prob.u0.copy()
    u[2, 40] = np.nan
    with pytest.raises(capi.DglmError, match="non-finite"):
        s.set_state(u)
    s.set_state(prob.u0)
    s.step(1)
    s.sync()
    s.close()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.gpu
@pytest.mark.parametrize("precision,kind,N", [("fp64", "pipe-dmma", 4), ("tf32x3", "tc-tmem", 4),
                                             ("bf16x3", "tc-tmem-bf16", 6)])
def test_bounded_waits_report_expiry(precision, kind, N):
    """Waits bounded to one cycle expire; the step reports DGLM_ERR_CUDA and
    the solver recovers once the bound is restored and a state is set."""
    prob = P.euler_sine(n=6, N=N, noise=1e-3, seed=4)       # 1,296 tets: 162 tiles of 8
    ref, _, _, _ = oracle.Oracle(prob).run(3)
    var = [v for v, d in capi.variants("euler", N, precision) if d.startswith(kind)][0]
    tol = 1e-12 if precision == "fp64" else 1e-6 if precision == "tf32x3" else 1e-5
    s = capi.Solver(prob, precision=precision, variant=var)
    s.set_wait_limit(1)
    s.step(1)
    with pytest.raises(capi.DglmError, match="bounded wait"):
        s.sync()
    s.set_wait_limit(0)
    s.set_state(prob.u0)
    s.step(3)
    s.sync()
    assert _rel(s.get_state(), ref) < tol
    s.close()
    fresh = capi.Solver(prob, precision=precision, variant=var)
    fresh.step(3)
    fresh.sync()
    assert _rel(fresh.get_state(), ref) < tol
    fresh.close()
