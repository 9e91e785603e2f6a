"""Drop-in for the reference's notebook launcher (dim3/src/python/
dglm_3d_launcher.py:10-463): same class names, constructor arguments,
method names, file layout and return values, so the notebook cells run with
only the import changed.

    from exadglm_b200.launcher import DGLM3DSingleGPU
    dg = DGLM3DSingleGPU(DGLM_DIR, WORK_DIR, N, Nvar, tmax, dglm_param, devid)
    dg.init_mesh(mesh_info)
    dg.make_work_dir()
    dg.save_to_binaries(matrix_order='f')
    dg.save_to_header([...]); dg.link_codes(filenames); dg.build([...])
    tstep, avg_dt, elapsed = dg.run('euler_nopad_main')
    l2 = dg.l2_error(u_ref, u_numeric)

Differences, by design: the reference builds its solver per run from
symlinked sources with nvcc and #defines (launcher :152-235, :459-462);
here ``build`` makes sure libdglm.so and the dglm_main driver exist
(compiled once for sm_100a, every order N <= 8) and ``run`` passes the
common.h parameters as flags.  ``dglm_dir`` is accepted and unused: the
operators and mesh come from this package.  The reference's ``gmsh`` mesh
type needs modules the reference does not ship and is not supported.
"""
from __future__ import annotations

import os
import re
import subprocess
import time

import numpy as np

from . import build as _build
from .datain import write_datain
from .mesh import Mesh3D, UniformBox
from .refelem import ref_element

PKG = os.path.dirname(os.path.abspath(__file__))


class DGLM3DBase:
    def __init__(self, dglm_dir, work_dir, N, Nvar, tmax, dglm_param):
        """Same arguments as the reference (dglm_3d_launcher.py:11-52):
        dglm_param keys CFL (0.8), gamma (1.4), tau_scale (1.2), interpN (2),
        dtype ('f8'; only 'f8' is supported)."""
        self.dglm_dir = os.path.abspath(dglm_dir) if dglm_dir else None
        self.work_dir = os.path.abspath(work_dir)
        self.N, self.Nvar, self.tmax = N, Nvar, tmax
        self.param = {"CFL": 0.8, "gamma": 1.4, "tau_scale": 1.2, "interpN": 2, "dtype": "f8"}
        self.param.update(dglm_param)
        if self.param["dtype"] != "f8":
            raise ValueError("only dtype 'f8' is supported (mixed precision is a solver mode)")
        if Nvar not in (1, 5):
            raise ValueError("Nvar must be 1 (advection) or 5 (Euler)")
        self.tet = ref_element(N, self.param["interpN"])
        self.op_ref = self.op_face = self.tet
        self.Np, self.Nfp, self.Nface = self.tet.Np, self.tet.Nfp, 4
        self.precision = "fp64"

    def init_mesh(self, mesh_info, verbose=1):
        """mesh_info = {'type': 'uniform', 'param': [nx, ny, nz, x1, x2, y1,
        y2, z1, z2, bc]} (launcher :361-381)."""
        if mesh_info["type"] != "uniform":
            raise NotImplementedError("only uniform meshes are supported (the reference's "
                                      "gmsh readers are not part of its release)")
        nx, ny, nz, x1, x2, y1, y2, z1, z2, *rest = mesh_info["param"]
        bc = rest[0] if rest else None
        box = UniformBox(nx, ny, nz, x1, x2, y1, y2, z1, z2, bc=bc)
        if verbose >= 1:
            print(f"Init uniform mesh: {mesh_info['param']}")
        self.mesh = Mesh3D(self.N, box, interpN=self.param["interpN"], high_order=True)
        self.Nelem = self.mesh.Nelem

    def make_work_dir(self):
        self.datain_dir = os.path.join(self.work_dir, "datain")
        self.dataout_dir = os.path.join(self.work_dir, "dataout")
        for d in (self.work_dir, self.datain_dir, self.dataout_dir):
            os.makedirs(d, exist_ok=True)

    def save_to_binaries(self, extra_arr_dict={}, matrix_order="c", verbose=1):
        """Write datain/*.bin (launcher :74-149); extra arrays such as u0,
        vx, vy, vz are written too and picked up by the driver."""
        arr = self.mesh.datain_arrays()
        arr.update(extra_arr_dict)
        self.matrix_order = matrix_order
        if verbose >= 1:
            print("Save DG arrays to *.bin files in WORK_DIR/datain/")
        write_datain(self.datain_dir, arr, matrix_order=matrix_order)

    def save_to_header(self, filename_list=[], extra_str_dict={}, extra_num_dict={}, verbose=1):
        """Writes common.h with the reference's #defines (launcher :152-205)
        for record keeping; the solver reads the same values as flags."""
        num = {"PI": 3.14159265358979323846, "TDIGIT": 7, "N": self.N, "NP": self.Np,
               "NFP": self.Nfp, "NFACE": 4, "NROT": 3, "NVAR": self.Nvar, "TMAX": self.tmax,
               "CFL": self.param["CFL"], "GAMMA": self.param["gamma"],
               "TAU_SCALE": self.param["tau_scale"]}
        num.update(extra_num_dict)
        lines = ["#ifndef COMMON_H", "#define COMMON_H", "", "#define REAL    double",
                 f'#define DATAIN  "{self.datain_dir}/"', f'#define DATAOUT "{self.dataout_dir}/"']
        lines += [f"#define {k} {v}" for k, v in extra_str_dict.items()]
        lines += [""] + [f"#define {k.ljust(6)} {v}" for k, v in num.items()] + ["", "#endif"]
        with open(os.path.join(self.work_dir, "common.h"), "w") as f:
            f.write("\n".join(lines) + "\n")
        if verbose >= 1:
            print("Save common.h files in WORK_DIR/")

    def link_codes(self, filename_list, verbose=1):
        """The reference symlinks its solver sources here (launcher
        :208-235); this solver is a prebuilt library, so only the requested
        names are recorded."""
        self.linked = list(filename_list)

    def check_mem_size(self, class_filename=None, verbose=1):
        """Device bytes of the solver's arrays for this mesh (the reference
        regex-estimates its cudaMalloc calls, utils/src/python/mem_size.py)."""
        K, Np, NF, nv = self.Nelem, self.Np, 4 * self.Nfp, self.Nvar
        vs = -(-K * Np // 32) * 32
        total = 8 * (3 * nv * vs + 9 * K + 4 * K * 5 + (3 * Np + NF) * (Np + 8)) \
            + 4 * (K * NF + 4 * K + NF)
        if nv == 1:
            total += 8 * 3 * vs
        if verbose >= 1:
            print(f"total bytes: {total / 1e6:.2f} MB")
        return total

    def build(self, filename_list=None, verbose=1):
        _build.build(verbose=verbose >= 2)

    def command(self, filename, full_state=False, restart_dir=None, restart_step=None):
        """The dglm_main command line for the executable name the notebook
        passes (advec_* or euler_*).  full_state writes every variable and
        the time file with each snapshot; restart_dir/restart_step continue
        from such a snapshot (neither is in the reference)."""
        physics = "advection" if os.path.basename(filename).startswith("advec") else "euler"
        if (physics == "euler") != (self.Nvar == 5):
            raise ValueError(f"{filename} does not match Nvar={self.Nvar}")
        if (restart_dir is None) != (restart_step is None):
            raise ValueError("restart_dir and restart_step go together")
        cmd = [_build.MAIN, "--datain", self.datain_dir, "--dataout", self.dataout_dir,
               "--physics", physics, "--tmax", repr(float(self.tmax)),
               "--cfl", repr(float(self.param["CFL"])),
               "--gamma", repr(float(self.param["gamma"])),
               "--tau-scale", repr(float(self.param["tau_scale"])),
               "--device", str(getattr(self, "devid", 0)),
               "--matrix-order", getattr(self, "matrix_order", "c"),
               "--precision", self.precision]
        if full_state:
            cmd.append("--full-state")
        if restart_dir is not None:
            cmd += ["--restart-dir", str(restart_dir), "--restart-step", str(int(restart_step))]
        return cmd

    def run(self, filename, omp_threads=None, verbose=1, full_state=False, restart_dir=None,
            restart_step=None):
        """Run the solver; returns (last_tstep, avg_dt, elapsed_time) parsed
        from its stdout as the reference does (launcher :283-325)."""
        cmd = self.command(filename, full_state, restart_dir, restart_step)
        if verbose >= 1:
            print(" ".join(cmd))
        t0 = time.perf_counter()
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
        elapsed = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"Error occurred: {r.stderr or 'non-zero exit code'}")
        if verbose >= 2:
            print(r.stdout)
        steps = re.findall(r"tstep=(\d+)", r.stdout)
        dts = re.findall(r"dt=([0-9.]+)", r.stdout)
        if not steps:
            return -1, -1, -1
        last, avg_dt = int(steps[-1]), np.array(dts, "f8").mean()
        if verbose >= 1:
            print(f"tstep={last}, dt={avg_dt:.5f}, elapsed_time={elapsed:.5f}")
        return last, avg_dt, elapsed

    def l2_error(self, ref_sol, numeric_sol, apply_sqrt=True):
        """Mass-weighted L2 error on the order-(N+interpN) nodes
        (launcher :328-355), vectorised."""
        K, Np, hNp = self.Nelem, self.Np, self.tet.high_Np
        un = np.asarray(numeric_sol).reshape(K, Np) @ self.tet.interpM.T
        E = np.asarray(ref_sol).reshape(K, hNp) - un
        s = np.sum(self.mesh.J * np.einsum("ki,ij,kj->k", E, self.tet.high_M, E))
        return np.sqrt(s) if apply_sqrt else s


class DGLM3DSingleCPU(DGLM3DBase):
    """Kept for the notebook import; the solver always runs on the GPU."""


class DGLM3DSingleGPU(DGLM3DSingleCPU):
    def __init__(self, dglm_dir, work_dir, N, Nvar, tmax, dglm_param, devid=0):
        self.devid = devid
        super().__init__(dglm_dir, work_dir, N, Nvar, tmax, dglm_param)
        self.pNP = ((self.Np - 1) // 32 + 1) * 32
        self.pNFF = ((self.Nface * self.Nfp - 1) // 32 + 1) * 32
