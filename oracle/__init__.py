"""ORACLE -- test infrastructure only.

Python access to the two CPU checkers of the DGLM hot path:

* :func:`lib` / :class:`Oracle` -- the C restatement in ``dglm_oracle.c``
  (built into ``oracle/liboracle.so``);
* :class:`RefSolver` -- the reference's own CPU solver compiled from its
  sources by ``build_ref.py`` into ``oracle/_ref/`` (present where that
  build ran).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
CFLAGS = ["-O3", "-std=c11", "-fopenmp", "-march=x86-64-v3", "-shared", "-fPIC"]

_lib = None


def build(force=False):
    src = os.path.join(HERE, "dglm_oracle.c")
    hdr = os.path.join(HERE, "dglm_oracle.h")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= max(os.path.getmtime(src), os.path.getmtime(hdr))):
        return LIB_PATH
    tmp = LIB_PATH + ".tmp"
    subprocess.run(["gcc", *CFLAGS, src, "-o", tmp, "-lm"], check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


class OrcMesh(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("N", "Np", "Nfp", "nvar", "K", "physics")] + \
               [(n, C.c_double) for n in ("cfl", "gamma", "tau_scale", "tmax")] + \
               [(n, C.c_void_p) for n in ("WDr", "WDs", "WDt", "LIFT", "rx", "ry", "rz", "sx",
                                          "sy", "sz", "tx", "ty", "tz", "Fscale", "nx", "ny",
                                          "nz", "EtoB", "vmapF", "vmapP", "Fmask", "vx", "vy",
                                          "vz")]


class OrcClock(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("tstep", C.c_int), ("last", C.c_int)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_calc_dt.restype = C.c_double
        L.orc_rhs.restype = C.c_double
        L.orc_run.restype = C.c_int
        L.orc_run.argtypes = [P, P, P, P, C.c_int, C.c_double, P]
        L.orc_lserk_stage.argtypes = [P, C.c_double, C.c_double, C.c_double, P, P, P]
        L.orc_num_threads.restype = C.c_int
        L.orc_run_record.argtypes = [P, P, P, C.c_int, P, P]
        L.orc_run_frozen.argtypes = [P, P, P, C.c_int, P, P]
        L.orc_rhs_adjoint.argtypes = [P, P, P, P, P]
        L.orc_adjoint.argtypes = [P, P, C.c_int, P, P, P]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Oracle:
    """The C restatement bound to one problem (mesh, parameters)."""

    def __init__(self, problem):
        self.p = problem
        arr = problem.datain_arrays()
        keep = {}

        def f64(name, a):
            keep[name] = np.ascontiguousarray(a, dtype=np.float64)
            return _ptr(keep[name])

        def i32(name, a):
            keep[name] = np.ascontiguousarray(a, dtype=np.int32)
            return _ptr(keep[name])

        m = OrcMesh()
        m.N, m.Np, m.Nfp = problem.N, problem.Np, problem.Nfp
        m.nvar, m.K = problem.nvar, problem.K
        m.physics = 1 if problem.physics == "euler" else 0
        m.cfl, m.gamma, m.tau_scale, m.tmax = problem.cfl, problem.gamma, problem.tau_scale, \
            problem.tmax
        for n in ("WDr", "WDs", "WDt", "LIFT", "rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty",
                  "tz", "Fscale", "nx", "ny", "nz"):
            setattr(m, n, f64(n, arr[n]))
        for n in ("EtoB", "vmapF", "vmapP", "Fmask"):
            setattr(m, n, i32(n, arr[n]))
        if problem.vel is not None:
            m.vx, m.vy, m.vz = f64("vx", problem.vel[0]), f64("vy", problem.vel[1]), \
                f64("vz", problem.vel[2])
        self.m, self._keep = m, keep
        self.L = lib()

    def _m(self):
        return C.byref(self.m)

    def run(self, nsteps, u=None, k=None, dt_fixed=0.0, clock=None):
        """nsteps LSERK steps from u (default u0).  Returns (u, k, clock,
        dt_hist)."""
        p = self.p
        u = np.array(p.u0 if u is None else u, dtype=np.float64, order="C").reshape(p.nvar, -1)
        k = np.zeros_like(u) if k is None else np.array(k, dtype=np.float64, order="C")
        clk = clock or OrcClock()
        hist = np.zeros(max(nsteps, 1))
        done = self.L.orc_run(self._m(), _ptr(u), _ptr(k), C.byref(clk), int(nsteps),
                              float(dt_fixed), _ptr(hist))
        return u, k, clk, hist[:done]

    def rhs(self, u=None):
        """One right-hand side: dict with maxv, tau, ub, fluxLM, fluxR/S/T,
        utmp and dt."""
        p = self.p
        u = np.ascontiguousarray(p.u0 if u is None else u, dtype=np.float64).reshape(p.nvar, -1)
        nF, nT, nV = p.K * 4, p.nvar * p.K * 4 * p.Nfp, p.nvar * p.K * p.Np
        out = {k: np.zeros(n) for k, n in (("maxv", nF), ("tau", nF), ("ub", nT),
                                             ("fluxLM", nT), ("fluxR", nV), ("fluxS", nV),
                                             ("fluxT", nV), ("utmp", nV))}
        dt = self.L.orc_rhs(self._m(), _ptr(u), *[_ptr(out[k]) for k in
                                                  ("maxv", "tau", "ub", "fluxLM", "fluxR",
                                                   "fluxS", "fluxT", "utmp")])
        out["dt"] = dt
        return out

    # ---- discrete adjoint (frozen dt and tau) ------------------------------

    def run_record(self, nsteps, u=None):
        """Forward run recording dt and tau per step.  Returns (u, dt_hist,
        tau_hist[nsteps, 4K])."""
        p = self.p
        u = np.array(p.u0 if u is None else u, dtype=np.float64, order="C").reshape(p.nvar, -1)
        k = np.zeros_like(u)
        dt = np.zeros(nsteps)
        tau = np.zeros((nsteps, 4 * p.K))
        self.L.orc_run_record(self._m(), _ptr(u), _ptr(k), int(nsteps), _ptr(dt), _ptr(tau))
        return u, dt, tau

    def run_frozen(self, u, dt_hist, tau_hist):
        """Forward run replaying recorded dt and tau (from k = 0)."""
        p = self.p
        u = np.array(u, dtype=np.float64, order="C").reshape(p.nvar, -1)
        k = np.zeros_like(u)
        dt = np.ascontiguousarray(dt_hist, dtype=np.float64)
        tau = np.ascontiguousarray(tau_hist, dtype=np.float64)
        self.L.orc_run_frozen(self._m(), _ptr(u), _ptr(k), len(dt), _ptr(dt), _ptr(tau))
        return u

    def rhs_frozen(self, u, tau):
        """R(u) with the face penalty tau given (update_ub, calc_fluxLM,
        calc_fluxes, update_rhs)."""
        p = self.p
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(p.nvar, -1)
        tau = np.ascontiguousarray(tau, dtype=np.float64)
        nT, nV = p.nvar * p.K * 4 * p.Nfp, p.nvar * p.K * p.Np
        ub, fLM = np.zeros(nT), np.zeros(nT)
        fR, fS, fT, out = np.zeros(nV), np.zeros(nV), np.zeros(nV), np.zeros(nV)
        L, m = self.L, self._m()
        L.orc_update_ub(m, _ptr(u), _ptr(ub))
        L.orc_calc_fluxLM(m, _ptr(u), _ptr(ub), _ptr(tau), _ptr(fLM))
        L.orc_calc_fluxes(m, _ptr(u), _ptr(fR), _ptr(fS), _ptr(fT))
        L.orc_update_rhs(m, _ptr(fR), _ptr(fS), _ptr(fT), _ptr(fLM), _ptr(out))
        return out.reshape(p.nvar, -1)

    def rhs_adjoint(self, u, tau, mu):
        """R'(u)^T mu with tau frozen."""
        p = self.p
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(p.nvar, -1)
        mu = np.ascontiguousarray(mu, dtype=np.float64).reshape(p.nvar, -1)
        tau = np.ascontiguousarray(tau, dtype=np.float64)
        lam = np.zeros_like(u)
        self.L.orc_rhs_adjoint(self._m(), _ptr(u), _ptr(tau), _ptr(mu), _ptr(lam))
        return lam

    def adjoint(self, u0, dt_hist, tau_hist, lam_T):
        """dJ/du(0) from dJ/du(T) = lam_T for the frozen run from u0."""
        p = self.p
        u0 = np.ascontiguousarray(u0, dtype=np.float64).reshape(p.nvar, -1)
        lam = np.array(lam_T, dtype=np.float64, order="C").reshape(p.nvar, -1)
        dt = np.ascontiguousarray(dt_hist, dtype=np.float64)
        tau = np.ascontiguousarray(tau_hist, dtype=np.float64)
        self.L.orc_adjoint(self._m(), _ptr(u0), len(dt), _ptr(dt), _ptr(tau), _ptr(lam))
        return lam

    @staticmethod
    def threads():
        return lib().orc_num_threads()


def rk_coefficients():
    a, b, c = (C.c_double * 5)(), (C.c_double * 5)(), (C.c_double * 5)()
    lib().orc_rk_coefficients(a, b, c)
    return np.array(a[:]), np.array(b[:]), np.array(c[:])


# ---------------------------------------------------------------------------
# the reference itself (oracle/_ref)
# ---------------------------------------------------------------------------

def host_has_avx512():
    """True when this host's CPU runs x86-64-v4 code (AVX-512 F/BW/CD/DQ/VL)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    return {"avx512f", "avx512bw", "avx512cd", "avx512dq",
                            "avx512vl"} <= flags
    except OSError:
        pass
    return False


def ref_march(physics, N):
    """The -march of the reference build that ref_lib_path loads here."""
    tag = "euler" if physics == "euler" else "advec"
    v4 = os.path.join(REF_DIR, f"libref_{tag}_N{N}_v4.so")
    return "x86-64-v4" if host_has_avx512() and os.path.exists(v4) else "x86-64-v3"


def ref_lib_path(physics, N):
    """The reference CPU solver built for this host: the AVX-512 build where
    the CPU has it (the launcher compiles with -march=native), else AVX2."""
    tag = "euler" if physics == "euler" else "advec"
    suffix = "_v4" if ref_march(physics, N) == "x86-64-v4" else ""
    return os.path.join(REF_DIR, f"libref_{tag}_N{N}{suffix}.so")


def ref_available(physics, N):
    return os.path.exists(ref_lib_path(physics, N))


class RefSolver:
    """The reference CPU solver (compiled from its sources) driven through
    oracle/ref_driver.cpp.  The datain files are written to a temporary
    directory in the CPU ('c') matrix order, as the reference expects.

    Each shared object keeps one global solver, so one RefSolver per
    (physics, N) is live at a time."""

    def __init__(self, problem, datain_dir=None):
        from exadglm_b200.datain import write_datain
        self.p = problem
        path = ref_lib_path(problem.physics, problem.N)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} (run oracle/build_ref.py where the reference lives)")
        L = C.CDLL(path)
        L.ref_open.restype = C.c_int
        L.ref_open.argtypes = [C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_double]
        L.ref_time.restype = C.c_double
        L.ref_last_dt.restype = C.c_double
        L.ref_rhs.restype = C.c_double
        L.ref_fetch.restype = C.c_long
        L.ref_fetch.argtypes = [C.c_char_p, C.c_void_p]
        self.L = L
        self._tmp = None
        if datain_dir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="dglm_ref_")
            datain_dir = self._tmp.name
            write_datain(datain_dir, problem.datain_arrays(), matrix_order="c")
        K = L.ref_open(datain_dir.encode(), problem.cfl, problem.gamma, problem.tau_scale,
                       problem.tmax)
        assert K == problem.K, (K, problem.K)
        if problem.vel is not None:
            v = np.ascontiguousarray(problem.vel, dtype=np.float64)
            L.ref_set_velocity(_ptr(v))
        self.set_state(problem.u0)

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.L.ref_set_state(_ptr(u))

    def get_state(self):
        u = np.zeros((self.p.nvar, self.p.K * self.p.Np))
        self.L.ref_get_state(_ptr(u))
        return u

    def run(self, nsteps):
        return self.L.ref_run(int(nsteps))

    def time(self):
        return self.L.ref_time(), self.L.ref_last_dt(), self.L.ref_tstep()

    def rhs(self):
        dt = self.L.ref_rhs()
        p = self.p
        nF, nT, nV = p.K * 4, p.nvar * p.K * 4 * p.Nfp, p.nvar * p.K * p.Np
        out = {"dt": dt}
        for k, n in (("maxv", nF), ("maxv_fs", nF), ("tau", nF), ("ub", nT), ("fluxLM", nT),
                     ("fluxR", nV), ("fluxS", nV), ("fluxT", nV), ("utmp", nV)):
            a = np.zeros(n)
            got = self.L.ref_fetch(k.encode(), _ptr(a))
            assert got == n, (k, got, n)
            out[k] = a
        return out

    def close(self):
        self.L.ref_close()
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None


# ---------------------------------------------------------------------------
# the reference GPU path (oracle/_ref/libref_gpu_euler_N4.so): the second
# baseline, the reference's own CUDA kernels and cuBLAS DGEMMs
# ---------------------------------------------------------------------------

def gpu_ref_lib_path(N=4):
    return os.path.join(REF_DIR, f"libref_gpu_euler_N{N}.so")


def gpu_ref_available(N=4):
    return os.path.exists(gpu_ref_lib_path(N))


class RefGpuSolver:
    """The reference Euler GPU solver (euler_nopad_*.cu with cuBLAS),
    compiled from its sources for one configuration (CFL, gamma and tau scale
    are compile-time constants there: build_ref.build_gpu_solver), driven
    through oracle/ref_gpu_driver.cu on the current CUDA device.  The datain
    files are written in the GPU ('f') matrix order.  One live instance per
    process (the shared object holds one global solver)."""

    def __init__(self, problem, datain_dir=None):
        from exadglm_b200.datain import write_datain
        if problem.physics != "euler":
            raise ValueError("the reference GPU build is the Euler path")
        self.p = problem
        path = gpu_ref_lib_path(problem.N)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} (run oracle/build_ref.py where the reference lives)")
        L = C.CDLL(path)
        L.ref_gpu_open.restype = C.c_int
        L.ref_gpu_open.argtypes = [C.c_char_p]
        for f in ("ref_gpu_cfl", "ref_gpu_gamma", "ref_gpu_tau_scale", "ref_gpu_time",
                  "ref_gpu_last_dt"):
            getattr(L, f).restype = C.c_double
        built = (L.ref_gpu_cfl(), L.ref_gpu_gamma(), L.ref_gpu_tau_scale())
        if built != (problem.cfl, problem.gamma, problem.tau_scale):
            raise ValueError(f"reference GPU build is for (CFL, gamma, tau) = {built}")
        self.L = L
        self._tmp = None
        if datain_dir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="dglm_refgpu_")
            datain_dir = self._tmp.name
            write_datain(datain_dir, problem.datain_arrays(), matrix_order="f")
        K = L.ref_gpu_open(datain_dir.encode())
        assert K == problem.K, (K, problem.K)
        self.set_state(problem.u0)

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert self.L.ref_gpu_set_state(_ptr(u)) == 0

    def get_state(self):
        u = np.zeros((self.p.nvar, self.p.K * self.p.Np))
        assert self.L.ref_gpu_get_state(_ptr(u)) == 0
        return u

    def run(self, nsteps):
        done = self.L.ref_gpu_run(int(nsteps))
        if done < 0:
            raise RuntimeError("reference GPU path: CUDA error")
        return done

    def time(self):
        return self.L.ref_gpu_time(), self.L.ref_gpu_last_dt(), self.L.ref_gpu_tstep()

    def close(self):
        self.L.ref_gpu_close()
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None
