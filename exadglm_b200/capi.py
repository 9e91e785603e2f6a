"""ctypes binding of libdglm.so (include/dglm.h).

The library is built in-tree by ``python -m exadglm_b200.build``; loading
fails loudly when it is missing -- there is no CPU fallback on this path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libdglm.so")

OK, ERR_INVALID, ERR_CUDA, ERR_NONFINITE, ERR_UNSUPPORTED, ERR_STATE, ERR_NOMEM, ERR_IO = range(8)
ADVECTION, EULER = 0, 1
PREC_FP64, PREC_TF32X3, PREC_BF16X3, PREC_BF16X6 = 0, 1, 2, 3
PRECISIONS = {"fp64": PREC_FP64, "tf32x3": PREC_TF32X3, "bf16x3": PREC_BF16X3,
              "bf16x6": PREC_BF16X6}

# every symbol include/dglm.h declares
EXPORTS = (
    "dglm_last_error", "dglm_abi_version", "dglm_order_supported", "dglm_create",
    "dglm_destroy", "dglm_set_stream", "dglm_upload_mesh", "dglm_set_state", "dglm_get_state",
    "dglm_step", "dglm_step_fixed_dt", "dglm_stage", "dglm_sync", "dglm_get_time", "dglm_set_time",
    "dglm_get_dt_history", "dglm_run_ensemble",
    "dglm_rhs", "dglm_kernel_launches", "dglm_device_bytes", "dglm_calc_maxv", "dglm_calc_dt",
    "dglm_update_tau", "dglm_update_ub", "dglm_calc_fluxLM", "dglm_calc_fluxes",
    "dglm_update_rhs", "dglm_lserk_stage", "dglm_variant_count", "dglm_variant_describe",
    "dglm_set_variant", "dglm_get_variant", "dglm_set_wait_limit",
    "dglm_set_compact_face_maps", "dglm_face_map_lists", "dglm_compact_face_maps",
    "dglm_adjoint_record", "dglm_adjoint_backward",
    "dglm_adjoint_replay", "dglm_adjoint_rhs", "dglm_adjoint_tape_bytes",
    "dglm_adjoint_record_capped", "dglm_adjoint_tape_plan", "dglm_adjoint_schedule",
    "dglm_calc_maxv_dt_static", "dglm_adjoint_variant_count", "dglm_adjoint_variant_describe",
    "dglm_adjoint_set_variant", "dglm_batch_create", "dglm_batch_add", "dglm_batch_finalize",
    "dglm_batch_step", "dglm_batch_sync", "dglm_batch_count", "dglm_batch_get_state",
    "dglm_batch_get_time", "dglm_batch_set_stream", "dglm_batch_kernel_launches",
    "dglm_batch_device_bytes", "dglm_batch_destroy",
)


class DglmError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"[dglm status {status}] {msg}")
        self.status = status


class Desc(C.Structure):
    _fields_ = [("N", C.c_int), ("physics", C.c_int), ("K", C.c_int), ("precision", C.c_int),
                ("cfl", C.c_double), ("gamma", C.c_double), ("tau_scale", C.c_double),
                ("tmax", C.c_double), ("device", C.c_int)]


_P = C.c_void_p
_MESH_FIELDS = ["WDr", "WDs", "WDt", "LIFT", "matrix_order", "rx", "ry", "rz", "sx", "sy", "sz",
                "tx", "ty", "tz", "Fscale", "nx", "ny", "nz", "EtoB", "vmapF", "vmapP", "Fmask",
                "vx", "vy", "vz"]


class MeshArrays(C.Structure):
    _fields_ = [(n, C.c_char if n == "matrix_order" else _P) for n in _MESH_FIELDS]


class BatchDesc(C.Structure):
    _fields_ = [("physics", C.c_int), ("cfl", C.c_double), ("tau_scale", C.c_double),
                ("tmax", C.c_double), ("device", C.c_int)]


_lib = None


def lib():
    """Load libdglm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m exadglm_b200.build` "
                               "(the CUDA library is the only implementation of this path)")
        L = C.CDLL(LIB_PATH)
        L.dglm_last_error.restype = C.c_char_p
        L.dglm_create.argtypes = [C.POINTER(Desc), C.POINTER(_P)]
        L.dglm_upload_mesh.argtypes = [_P, C.POINTER(MeshArrays)]
        L.dglm_set_state.argtypes = [_P, _P, C.c_int]
        L.dglm_get_state.argtypes = [_P, _P, C.c_int]
        L.dglm_step.argtypes = [_P, C.c_int]
        L.dglm_step_fixed_dt.argtypes = [_P, C.c_int, C.c_double]
        L.dglm_stage.argtypes = [_P, C.c_int, C.c_double]
        L.dglm_set_stream.argtypes = [_P, _P]
        L.dglm_sync.argtypes = [_P]
        L.dglm_destroy.argtypes = [_P]
        L.dglm_get_time.argtypes = [_P, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_int)]
        L.dglm_set_time.argtypes = [_P, C.c_double, C.c_int]
        L.dglm_run_ensemble.argtypes = [_P, C.c_int, _P, _P, C.c_int, C.POINTER(C.c_int)]
        L.dglm_get_dt_history.argtypes = [_P, C.c_int, C.c_int, _P]
        L.dglm_rhs.argtypes = [_P, _P, _P]
        L.dglm_variant_describe.argtypes = [C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_size_t]
        L.dglm_set_variant.argtypes = [_P, C.c_int]
        L.dglm_get_variant.argtypes = [_P]
        L.dglm_set_wait_limit.argtypes = [_P, C.c_longlong]
        L.dglm_set_compact_face_maps.argtypes = [_P, C.c_int]
        L.dglm_face_map_lists.argtypes = [_P]
        L.dglm_compact_face_maps.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_int,
                                             C.POINTER(C.c_int)]
        L.dglm_kernel_launches.argtypes = [_P]
        L.dglm_kernel_launches.restype = C.c_long
        L.dglm_device_bytes.argtypes = [_P]
        L.dglm_device_bytes.restype = C.c_size_t
        D, I = C.c_double, C.c_int
        L.dglm_calc_maxv.argtypes = [I, I, I, D, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.dglm_calc_dt.argtypes = [I, I, D, _P, _P, _P]
        L.dglm_update_tau.argtypes = [I, D, _P, _P, _P, _P]
        L.dglm_update_ub.argtypes = [I, I, I, _P, _P, _P, _P, _P]
        L.dglm_calc_fluxLM.argtypes = [I, I, I, D, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                       _P, _P]
        L.dglm_calc_fluxes.argtypes = [I, I, I, D, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.dglm_update_rhs.argtypes = [I, I, I, _P, _P, _P, _P, C.c_char, _P, _P, _P, _P, _P, _P]
        L.dglm_lserk_stage.argtypes = [I, I, I, D, D, D, _P, _P, _P, _P]
        L.dglm_calc_maxv_dt_static.argtypes = [I, I, I, D, D, _P, _P, _P, _P, _P, _P, _P, _P,
                                               _P]
        L.dglm_adjoint_record.argtypes = [_P, I, I]
        L.dglm_adjoint_backward.argtypes = [_P, _P, _P, I]
        L.dglm_adjoint_replay.argtypes = [_P]
        L.dglm_adjoint_rhs.argtypes = [_P, _P, _P, _P]
        L.dglm_adjoint_tape_bytes.argtypes = [_P, C.POINTER(C.c_size_t)]
        L.dglm_adjoint_record_capped.argtypes = [_P, I, C.c_size_t]
        L.dglm_adjoint_tape_plan.argtypes = [_P, C.POINTER(I), C.POINTER(I),
                                             C.POINTER(C.c_longlong)]
        L.dglm_adjoint_schedule.argtypes = [I, I, I, I, _P, I, C.POINTER(I), _P, I, C.POINTER(I),
                                            C.POINTER(C.c_longlong)]
        L.dglm_adjoint_variant_describe.argtypes = [I, I, I, C.c_char_p, C.c_size_t]
        L.dglm_batch_create.argtypes = [C.POINTER(BatchDesc), C.POINTER(_P)]
        L.dglm_batch_add.argtypes = [_P, I, I, C.POINTER(MeshArrays), _P, _P, C.POINTER(I)]
        L.dglm_batch_finalize.argtypes = [_P]
        L.dglm_batch_step.argtypes = [_P, I]
        L.dglm_batch_sync.argtypes = [_P]
        L.dglm_batch_count.argtypes = [_P]
        L.dglm_batch_get_state.argtypes = [_P, I, _P, I]
        L.dglm_batch_get_time.argtypes = [_P, I, C.POINTER(D), C.POINTER(D), C.POINTER(I)]
        L.dglm_batch_set_stream.argtypes = [_P, _P]
        L.dglm_batch_kernel_launches.argtypes = [_P]
        L.dglm_batch_kernel_launches.restype = C.c_long
        L.dglm_batch_device_bytes.argtypes = [_P]
        L.dglm_batch_device_bytes.restype = C.c_size_t
        L.dglm_batch_destroy.argtypes = [_P]
        L.dglm_adjoint_set_variant.argtypes = [_P, I]
        _lib = L
    return _lib


def check(status):
    if status != OK:
        raise DglmError(status, lib().dglm_last_error().decode())


def ptr_table(ptrs):
    """HOST array of device (or host) pointers, as the per-variable tables of
    the C ABI expect."""
    arr = (C.c_void_p * len(ptrs))(*[C.c_void_p(int(p)) for p in ptrs])
    return arr


def variant_precision(desc):
    """Precision mode of a variant from its description."""
    for prec in ("tf32x3", "bf16x3", "bf16x6"):
        if desc.startswith(("tcgen05-" + prec, "mma16-" + prec, "pipe-mma16-" + prec)):
            return prec
    # split TF32 / BF16 with all four part products (the tensor-memory
    # operator kernels)
    if desc.startswith("tc-tmem-tf32"):
        return "tf32x3"
    if desc.startswith("tc-tmem-bf16"):
        return "bf16x3"
    return "fp64"


def variants(physics, N, precision=None):
    """Descriptions of the compiled stage-kernel variants for (physics, N),
    indexed by variant number; with `precision`, the indices of that mode
    only are returned as (index, description) pairs."""
    L = lib()
    ph = EULER if physics == "euler" else ADVECTION
    out = []
    for i in range(L.dglm_variant_count(ph, N)):
        buf = C.create_string_buffer(128)
        check(L.dglm_variant_describe(ph, N, i, buf, 128))
        out.append(buf.value.decode())
    if precision is None:
        return out
    return [(i, d) for i, d in enumerate(out) if variant_precision(d) == precision]


def adjoint_schedule(nsteps, leaf, slots, prestored=True):
    """The binomial checkpointing schedule (host only): (spine, actions,
    advance_steps); spine[q] = chunk held by slot q after the recording,
    actions = rows (kind, src, chunk, count, dst), kind 0 advance, 1 reverse."""
    L = lib()
    n = (int(nsteps) + int(leaf) - 1) // int(leaf)
    cap_a = 4 * n * n + 16
    spine = np.zeros(n + 1, dtype=np.int32)
    acts = np.zeros((cap_a, 5), dtype=np.int32)
    ns, na, adv = C.c_int(), C.c_int(), C.c_longlong()
    check(L.dglm_adjoint_schedule(int(nsteps), int(leaf), int(slots), int(bool(prestored)),
                                  spine.ctypes.data, len(spine), C.byref(ns), acts.ctypes.data,
                                  cap_a, C.byref(na), C.byref(adv)))
    return spine[:ns.value].copy(), acts[:na.value].copy(), adv.value


def compact_face_maps(vmapP, Np, Nfp, max_lists=256):
    """The compact form of a vmapP (K x 4 x Nfp) that
    Solver.set_compact_face_maps builds (host only): (etoe, code, lists) with
    vmapP[e, f, j] = etoe[e, f] Np + lists[code[e, f], j]."""
    L = lib()
    vm = np.ascontiguousarray(vmapP, dtype=np.int32).reshape(-1, 4, Nfp)
    K = vm.shape[0]
    etoe = np.zeros((K, 4), dtype=np.int32)
    code = np.zeros((K, 4), dtype=np.uint8)
    lists = np.zeros((max(int(max_lists), 1), Nfp), dtype=np.int32)
    n = C.c_int()
    check(L.dglm_compact_face_maps(K, int(Np), int(Nfp), vm.ctypes.data, etoe.ctypes.data,
                                   code.ctypes.data, lists.ctypes.data, int(max_lists),
                                   C.byref(n)))
    return etoe, code, lists[:n.value].copy()


def adjoint_variants(physics, N):
    """Descriptions of the adjoint stage-kernel tile shapes for (physics, N)."""
    L = lib()
    ph = EULER if physics == "euler" else ADVECTION
    out = []
    for i in range(L.dglm_adjoint_variant_count(ph, N)):
        buf = C.create_string_buffer(128)
        check(L.dglm_adjoint_variant_describe(ph, N, i, buf, 128))
        out.append(buf.value.decode())
    return out


def _np_ptr(a):
    return C.c_void_p(a.ctypes.data)


def mesh_arrays(problem, arr, matrix_order="c", with_velocity=True):
    """A MeshArrays struct over contiguous copies of the problem's datain
    arrays; returns (struct, the arrays it points into)."""
    keep = {}

    def f64(name, a, order="C"):
        keep[name] = np.ascontiguousarray(np.asarray(a, np.float64).ravel(order))
        return keep[name].ctypes.data

    def i32(name, a):
        keep[name] = np.ascontiguousarray(np.asarray(a, np.int32).ravel())
        return keep[name].ctypes.data

    m = MeshArrays()
    m.matrix_order = matrix_order.encode()
    order = "F" if matrix_order == "f" else "C"
    for n in ("WDr", "WDs", "WDt", "LIFT"):
        setattr(m, n, f64(n, arr[n], order))
    for n in ("rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz", "Fscale", "nx", "ny", "nz"):
        setattr(m, n, f64(n, arr[n]))
    for n in ("EtoB", "vmapF", "vmapP", "Fmask"):
        setattr(m, n, i32(n, arr[n]))
    if with_velocity and problem.vel is not None:
        m.vx, m.vy, m.vz = (f64(n, problem.vel[i]) for i, n in enumerate(("vx", "vy", "vz")))
    return m, keep


class Solver:
    """A solver handle for one problem (see :mod:`exadglm_b200.problem`).

    ``state`` arrays are numpy (nvar, K*Np) on the host, or lists of device
    pointers for the on-device variants."""

    def __init__(self, problem, precision="fp64", device=0, matrix_order="c", arrays=None,
                 variant=None):
        """variant: stage-kernel tile shape; None takes the tuned choice for
        this device from exadglm_b200/tuned.json when present, a negative
        value the library default (the first variant of the precision)."""
        self.p = problem
        L = lib()
        d = Desc()
        d.N, d.K = problem.N, problem.K
        d.physics = EULER if problem.physics == "euler" else ADVECTION
        d.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        self.precision = {v: k for k, v in PRECISIONS.items()}[d.precision]
        d.cfl, d.gamma, d.tau_scale, d.tmax = problem.cfl, problem.gamma, problem.tau_scale, \
            problem.tmax
        d.device = device
        h = _P()
        check(L.dglm_create(C.byref(d), C.byref(h)))
        self.h, self.L = h, L
        arr = arrays if arrays is not None else problem.datain_arrays()
        m, self._keep = mesh_arrays(problem, arr, matrix_order)
        check(L.dglm_upload_mesh(h, C.byref(m)))
        if variant is None:
            from .tune import cached_variant
            variant = cached_variant(problem.physics, problem.N, self.precision, device)
        if variant is not None and variant >= 0:
            self.set_variant(variant)
        self.set_state(problem.u0)

    # -- state ------------------------------------------------------------
    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.p.nvar, -1)
        self._u_host = u
        check(self.L.dglm_set_state(self.h, ptr_table([u[v].ctypes.data for v in range(len(u))]),
                                    0))

    def set_state_ptrs(self, ptrs, on_device):
        check(self.L.dglm_set_state(self.h, ptr_table(ptrs), int(on_device)))

    def get_state_ptrs(self, ptrs, on_device):
        check(self.L.dglm_get_state(self.h, ptr_table(ptrs), int(on_device)))

    def set_state_device(self, ptrs):
        check(self.L.dglm_set_state(self.h, ptr_table(ptrs), 1))

    def get_state(self):
        out = np.empty((self.p.nvar, self.p.K * self.p.Np))
        check(self.L.dglm_get_state(self.h, ptr_table([out[v].ctypes.data
                                                        for v in range(len(out))]), 0))
        return out

    def get_state_device(self, ptrs):
        check(self.L.dglm_get_state(self.h, ptr_table(ptrs), 1))

    # -- time stepping ----------------------------------------------------
    def step(self, nsteps=1, dt=None):
        if dt is None:
            check(self.L.dglm_step(self.h, int(nsteps)))
        else:
            check(self.L.dglm_step_fixed_dt(self.h, int(nsteps), float(dt)))

    def stage(self, stage, dt):
        check(self.L.dglm_stage(self.h, int(stage), float(dt)))

    def sync(self):
        check(self.L.dglm_sync(self.h))

    def time(self):
        t, dt, ts = C.c_double(), C.c_double(), C.c_int()
        check(self.L.dglm_get_time(self.h, C.byref(t), C.byref(dt), C.byref(ts)))
        return t.value, dt.value, ts.value

    def set_time(self, t, tstep):
        """Continue a saved run: time and step counter after set_state."""
        check(self.L.dglm_set_time(self.h, float(t), int(tstep)))

    def run_ensemble_ptrs(self, in_ptrs, out_ptrs, nsteps):
        """dglm_run_ensemble: member i reads the host fields in_ptrs[i] (nvar
        pointers) and, after nsteps steps from t = 0, writes out_ptrs[i]; the
        host<->device copies overlap the compute (page-locked memory).
        Returns the index of the first non-finite member (an error is raised
        with it) or -1."""
        count = len(in_ptrs)
        if len(out_ptrs) != count:
            raise ValueError("run_ensemble: as many outputs as inputs")
        tins = [ptr_table(p) for p in in_ptrs]
        touts = [ptr_table(p) for p in out_ptrs]
        tin = (C.c_void_p * max(count, 1))(*[C.cast(t, C.c_void_p) for t in tins])
        tout = (C.c_void_p * max(count, 1))(*[C.cast(t, C.c_void_p) for t in touts])
        bad = C.c_int(-1)
        st = self.L.dglm_run_ensemble(self.h, count, tin, tout, int(nsteps), C.byref(bad))
        self.first_bad = bad.value
        check(st)
        return bad.value

    def run_ensemble(self, states, nsteps=1):
        """Numpy front end: states is a sequence of (nvar, K*Np) arrays;
        returns the evolved states (pageable memory: correct, not overlapped)."""
        ins = [np.ascontiguousarray(u, dtype=np.float64).reshape(self.p.nvar, -1) for u in states]
        outs = [np.empty_like(u) for u in ins]
        self.run_ensemble_ptrs([[u[v].ctypes.data for v in range(self.p.nvar)] for u in ins],
                               [[o[v].ctypes.data for v in range(self.p.nvar)] for o in outs],
                               nsteps)
        return outs

    def save_full_state(self, dirpath, print_interval=0):
        """Write the current state and time as a full-state snapshot (the
        format of ``dglm_main --full-state``); returns the step number."""
        from .datain import write_full_state
        t, _, tstep = self.time()
        write_full_state(dirpath, tstep, self.p.physics, self.get_state(), t, print_interval)
        return tstep

    def restart(self, dirpath, tstep):
        """Continue from a full-state snapshot: set_state + set_time."""
        from .datain import read_full_state
        u, t, step, _ = read_full_state(dirpath, tstep, self.p.physics,
                                        n=self.p.K * self.p.Np)
        self.set_state(u)
        self.set_time(t, step)
        return t, step

    def dt_history(self, first, count):
        out = np.zeros(count)
        check(self.L.dglm_get_dt_history(self.h, int(first), int(count), _np_ptr(out)))
        return out

    def rhs_device(self, u_ptrs, rhs_ptrs):
        check(self.L.dglm_rhs(self.h, ptr_table(u_ptrs), ptr_table(rhs_ptrs)))

    # -- discrete adjoint (FP64; dt and tau frozen at the recorded values) --
    def adjoint_record(self, nsteps, checkpoint_every=50):
        """nsteps CFL steps from the current state, recording the tape."""
        check(self.L.dglm_adjoint_record(self.h, int(nsteps), int(checkpoint_every)))

    def adjoint_record_capped(self, nsteps, max_bytes):
        """nsteps CFL steps from the current state, recording a tape of at
        most max_bytes of device memory (binomial checkpointing)."""
        check(self.L.dglm_adjoint_record_capped(self.h, int(nsteps), int(max_bytes)))

    def adjoint_tape_plan(self):
        """(leaf steps, checkpoint slots, forward steps the next backward
        pass recomputes) of the recorded tape."""
        leaf, slots, adv = C.c_int(), C.c_int(), C.c_longlong()
        check(self.L.dglm_adjoint_tape_plan(self.h, C.byref(leaf), C.byref(slots),
                                            C.byref(adv)))
        return leaf.value, slots.value, adv.value

    def adjoint_backward(self, lam_T):
        """(du_T/du_0)^T lam_T for the recorded run (numpy in, numpy out)."""
        lam_T = np.ascontiguousarray(lam_T, dtype=np.float64).reshape(self.p.nvar, -1)
        out = np.empty_like(lam_T)
        check(self.L.dglm_adjoint_backward(
            self.h, ptr_table([lam_T[v].ctypes.data for v in range(len(lam_T))]),
            ptr_table([out[v].ctypes.data for v in range(len(out))]), 0))
        return out

    def adjoint_backward_device(self, lam_T_ptrs, lam_0_ptrs):
        check(self.L.dglm_adjoint_backward(self.h, ptr_table(lam_T_ptrs), ptr_table(lam_0_ptrs),
                                           1))

    def adjoint_replay(self):
        """The recorded run from the current state with recorded dt and tau."""
        check(self.L.dglm_adjoint_replay(self.h))

    def adjoint_rhs_device(self, u_ptrs, mu_ptrs, out_ptrs):
        check(self.L.dglm_adjoint_rhs(self.h, ptr_table(u_ptrs), ptr_table(mu_ptrs),
                                      ptr_table(out_ptrs)))

    def adjoint_set_variant(self, v):
        check(self.L.dglm_adjoint_set_variant(self.h, int(v)))

    def adjoint_tape_bytes(self):
        n = C.c_size_t()
        check(self.L.dglm_adjoint_tape_bytes(self.h, C.byref(n)))
        return int(n.value)

    def set_stream(self, stream_ptr):
        check(self.L.dglm_set_stream(self.h, C.c_void_p(int(stream_ptr))))

    def set_variant(self, v):
        check(self.L.dglm_set_variant(self.h, int(v)))

    def variant(self):
        return int(self.L.dglm_get_variant(self.h))

    def set_wait_limit(self, cycles):
        """Bound (SM clock cycles) of the hand-off waits of the pipelined
        stage kernels; 0 restores the default (about one second)."""
        check(self.L.dglm_set_wait_limit(self.h, int(cycles)))

    def set_compact_face_maps(self, on=True):
        """Neighbour node indices from compact face maps (neighbour element
        and a one-byte node-list code per face) instead of vmapP in the
        persistent stage kernels; bit for bit the same results."""
        check(self.L.dglm_set_compact_face_maps(self.h, 1 if on else 0))

    def face_map_lists(self):
        """Distinct face node lists of the compact face maps (0 before built)."""
        return int(self.L.dglm_face_map_lists(self.h))

    def kernel_launches(self):
        return int(self.L.dglm_kernel_launches(self.h))

    def device_bytes(self):
        return int(self.L.dglm_device_bytes(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.L.dglm_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchSolver:
    """Many independent advection problems (orders 2..6, constant velocity
    each) advanced together by one persistent launch per LSERK stage.

    ``problems`` share cfl, tau_scale and tmax (taken from the first)."""

    def __init__(self, problems, device=0, cfl=None, tau_scale=None, tmax=None):
        L = lib()
        p0 = problems[0]
        d = BatchDesc()
        d.physics = ADVECTION
        d.cfl = p0.cfl if cfl is None else cfl
        d.tau_scale = p0.tau_scale if tau_scale is None else tau_scale
        d.tmax = p0.tmax if tmax is None else tmax
        d.device = device
        h = _P()
        check(L.dglm_batch_create(C.byref(d), C.byref(h)))
        self.h, self.L, self.problems = h, L, list(problems)
        try:
            for p in problems:
                if p.physics != "advection" or p.vel is None:
                    raise ValueError("BatchSolver: advection problems with a velocity only")
                v = np.asarray(p.vel, np.float64)
                vel = np.ascontiguousarray(v[:, 0])
                if not (v.min(axis=1) == v.max(axis=1)).all():
                    raise ValueError("BatchSolver: each problem's velocity must be constant")
                m, keep = mesh_arrays(p, p.datain_arrays(), with_velocity=False)
                u0 = np.ascontiguousarray(np.asarray(p.u0, np.float64).ravel())
                idx = C.c_int()
                check(L.dglm_batch_add(h, p.N, p.K, C.byref(m), u0.ctypes.data, vel.ctypes.data,
                                       C.byref(idx)))
            check(L.dglm_batch_finalize(h))
        except Exception:
            self.close()
            raise

    def step(self, nsteps=1):
        check(self.L.dglm_batch_step(self.h, int(nsteps)))

    def sync(self):
        check(self.L.dglm_batch_sync(self.h))

    def get_state(self, i):
        p = self.problems[i]
        out = np.empty(p.K * p.Np)
        check(self.L.dglm_batch_get_state(self.h, int(i), out.ctypes.data, 0))
        return out

    def time(self, i):
        t, dt, ts = C.c_double(), C.c_double(), C.c_int()
        check(self.L.dglm_batch_get_time(self.h, int(i), C.byref(t), C.byref(dt), C.byref(ts)))
        return t.value, dt.value, ts.value

    def set_stream(self, stream_ptr):
        check(self.L.dglm_batch_set_stream(self.h, C.c_void_p(int(stream_ptr))))

    def kernel_launches(self):
        return int(self.L.dglm_batch_kernel_launches(self.h))

    def device_bytes(self):
        return int(self.L.dglm_batch_device_bytes(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.L.dglm_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
