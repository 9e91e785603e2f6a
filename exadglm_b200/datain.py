"""The reference's file formats: ``datain/*.bin`` inputs and ``dataout``
snapshots.

Every file is a raw little-endian array with no header
(utils/src/cpp/io.cpp:7-29).  Integer arrays are int32, real arrays float64.
The four operator matrices are stored 'c' (row-major) for the CPU solver and
'f' (column-major) for the cuBLAS GPU solver (dglm_3d_launcher.py:138-147);
every other array is stored flat in C order.  Snapshots are
``u_NNNNNNN.bin`` (advection) and ``u1_NNNNNNN.bin`` (Euler density) with a
7-digit zero-padded step (advec_data.cpp:287-291, euler_data.cpp:287-294).

Full state (not in the reference, which writes only the first variable and
cannot restart): the other Euler variables as ``u2_`` .. ``u5_NNNNNNN.bin``
and ``t_NNNNNNN.bin``, three float64 values (t, the step number, the print
interval; 0 when unknown).  ``dglm_main --full-state`` writes the same bytes.
"""
from __future__ import annotations

import os

import numpy as np

INT_ARRAYS = ("dim", "EtoB", "vmapP", "vmapF", "Fmask")
OPERATORS = ("WDr", "WDs", "WDt", "LIFT")
ELEM_ARRAYS = ("rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz")
FACE_ARRAYS = ("Fscale", "nx", "ny", "nz")
NODE_ARRAYS = ("px", "py", "pz")
ALL_ARRAYS = INT_ARRAYS + OPERATORS + ELEM_ARRAYS + FACE_ARRAYS + NODE_ARRAYS
TDIGIT = 7


def write_datain(dirpath, arrays, matrix_order="c"):
    """Write a dict of arrays (names as in ALL_ARRAYS, plus extras) as
    ``dirpath/<name>.bin``."""
    os.makedirs(dirpath, exist_ok=True)
    for name, arr in arrays.items():
        arr = np.asarray(arr)
        if name in INT_ARRAYS:
            arr = arr.astype(np.int32)
        elif arr.dtype.kind == "f":
            arr = arr.astype(np.float64)
        flat = arr.ravel(matrix_order) if name in OPERATORS else arr.ravel()
        flat.tofile(os.path.join(dirpath, f"{name}.bin"))


def order_from_np(Np):
    for N in range(0, 64):
        if (N + 1) * (N + 2) * (N + 3) // 6 == Np:
            return N
    raise ValueError(f"{Np} is not a tetrahedral node count")


def read_datain(dirpath, matrix_order="c"):
    """Read a datain directory back.  N is inferred from the size of WDr.bin.
    Returns (N, dict of arrays shaped like the launcher's, operators in
    (rows, cols) form)."""
    def rd(name, dtype):
        path = os.path.join(dirpath, f"{name}.bin")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        return np.fromfile(path, dtype=dtype)

    K = int(rd("dim", np.int32)[0])
    wdr = rd("WDr", np.float64)
    Np = int(round(np.sqrt(wdr.size)))
    if Np * Np != wdr.size:
        raise ValueError("WDr.bin is not square")
    N = order_from_np(Np)
    Nfp = (N + 1) * (N + 2) // 2
    out = {"dim": np.array([K], np.int32)}
    for name in OPERATORS:
        cols = Np if name != "LIFT" else 4 * Nfp
        a = rd(name, np.float64)
        if a.size != Np * cols:
            raise ValueError(f"{name}.bin has {a.size} values, expected {Np * cols}")
        out[name] = a.reshape((Np, cols), order="C" if matrix_order == "c" else "F")
    shapes = {"EtoB": (K, 4), "vmapF": (K, 4), "vmapP": (K, 4, Nfp), "Fmask": (4, Nfp)}
    for name, shp in shapes.items():
        a = rd(name, np.int32)
        if a.size != int(np.prod(shp)):
            raise ValueError(f"{name}.bin has {a.size} values, expected {int(np.prod(shp))}")
        out[name] = a.reshape(shp)
    for name in ELEM_ARRAYS:
        out[name] = rd(name, np.float64).reshape(K)
    for name in FACE_ARRAYS:
        out[name] = rd(name, np.float64).reshape(K, 4)
    for name in NODE_ARRAYS:
        out[name] = rd(name, np.float64).reshape(K, Np)
    return N, out


def snapshot_name(tstep, physics):
    s = str(int(tstep))
    prefix = "u1_" if physics == "euler" else "u_"
    return prefix + "0" * (TDIGIT - len(s)) + s + ".bin"


def write_snapshot(dirpath, tstep, physics, u_first_var):
    os.makedirs(dirpath, exist_ok=True)
    path = os.path.join(dirpath, snapshot_name(tstep, physics))
    np.ascontiguousarray(u_first_var, dtype=np.float64).tofile(path)
    return path


def _step(tstep):
    s = str(int(tstep))
    if int(tstep) < 0 or len(s) > TDIGIT:
        raise ValueError(f"step {tstep} does not fit the {TDIGIT}-digit snapshot names")
    return "0" * (TDIGIT - len(s)) + s


def field_name(v, tstep, physics):
    """Snapshot file of variable v (0-based): ``u_`` (advection),
    ``u1_`` .. ``u5_`` (Euler)."""
    if physics == "euler":
        if not 0 <= v < 5:
            raise ValueError("Euler has variables 0..4")
        return f"u{v + 1}_" + _step(tstep) + ".bin"
    if v != 0:
        raise ValueError("advection has one variable")
    return "u_" + _step(tstep) + ".bin"


def time_name(tstep):
    return "t_" + _step(tstep) + ".bin"


def write_full_state(dirpath, tstep, physics, u, t, print_interval=0):
    """Every variable of u (nvar, K*Np) and the time file of step tstep."""
    nvar = 5 if physics == "euler" else 1
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(nvar, -1)
    os.makedirs(dirpath, exist_ok=True)
    for v in range(nvar):
        u[v].tofile(os.path.join(dirpath, field_name(v, tstep, physics)))
    np.array([t, tstep, print_interval], dtype=np.float64).tofile(
        os.path.join(dirpath, time_name(tstep)))


def read_full_state(dirpath, tstep, physics, n=None):
    """(u (nvar, n), t, tstep, print_interval) of a full-state snapshot;
    n = K*Np is checked when given."""
    nvar = 5 if physics == "euler" else 1
    fields = []
    for v in range(nvar):
        f = np.fromfile(os.path.join(dirpath, field_name(v, tstep, physics)), dtype=np.float64)
        if n is not None and f.size != n:
            raise ValueError(f"{field_name(v, tstep, physics)} holds {f.size} values, "
                             f"expected {n}")
        if fields and f.size != fields[0].size:
            raise ValueError("the fields of the snapshot differ in size")
        fields.append(f)
    tt = np.fromfile(os.path.join(dirpath, time_name(tstep)), dtype=np.float64)
    if tt.size != 3 or int(round(tt[1])) != int(tstep):
        raise ValueError(f"{time_name(tstep)} is not the time file of step {tstep}")
    return np.stack(fields), float(tt[0]), int(round(tt[1])), int(round(tt[2]))


def full_state_steps(dirpath, physics):
    """Steps of dirpath that have every field and the time file."""
    nvar = 5 if physics == "euler" else 1
    steps = []
    for name in sorted(os.listdir(dirpath)):
        if name.startswith("t_") and name.endswith(".bin") and name[2:-4].isdigit():
            k = int(name[2:-4])
            if all(os.path.exists(os.path.join(dirpath, field_name(v, k, physics)))
                   for v in range(nvar)):
                steps.append(k)
    return steps
