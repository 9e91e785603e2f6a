"""Build recipe for ``oracle/_ref/``: the reference's own code, compiled from
its sources where they lie in the reference tree (nothing is copied).

Products (all git-ignored, they travel with the working tree):

* ``_ref/libref_{euler,advec}_N{n}.so`` -- the reference CPU single-partition
  solver (dim3/src/cpp/{euler,advec}_{data,dglm,time}.cpp, plus
  utils/src/cpp/io.cpp), compiled the way its launcher does
  (dglm_3d_launcher.py:392: ``g++ -O3 -std=c++11 -fopenmp -march=native``),
  with the generated ``common.h`` written here.  ``native`` would tie the
  library to this machine's CPU, so two builds are made instead: one for
  ``-march=x86-64-v3`` (AVX2) and one for ``-march=x86-64-v4`` (AVX-512,
  suffix ``_v4``); oracle.ref_lib_path loads the v4 build on hosts whose
  CPU has AVX-512 -- the closest portable stand-in for ``native``.
  ``ref_driver.cpp`` wraps its ``runRK`` in a fixed-step C entry point.
  ``CFL``, ``GAMMA``, ``TAU_SCALE`` and ``TMAX`` become run-time globals so
  one build serves every configuration of an order N; ``N``, ``NP``, ``NFP``,
  ``NVAR`` stay compile-time as in the reference.
* ``_ref/libref_gpu_euler_N4.so`` -- the reference GPU path
  (dim3/src/cuda/euler_nopad_{data_host,data_dev,dglm,time}.cu, CUDA kernels
  and cuBLAS batched DGEMMs) for the benchmark workload (CFL 0.4, gamma 1.4,
  tau scale 1.2), compiled for sm_100a; ``ref_gpu_driver.cu`` wraps its
  ``runRK``.  The second baseline of the benchmark.
* ``_ref/mesh_3d_cpp*.so``, ``_ref/uniform_3d_single_cpp*.so`` -- the
  reference's pybind11 mesh cores rebuilt from dim3/src/cpp (used only to
  generate golden fixtures in a container that holds the reference).

Usage: ``python oracle/build_ref.py [--orders 1-6]``.  Exits quietly with a
message when the reference tree is absent.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference tree: $DGLM_REFERENCE_ROOT, else a "reference" directory
# beside the repository
REF = os.environ.get("DGLM_REFERENCE_ROOT",
                     os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
CXXFLAGS = ["-O3", "-std=c++11", "-fopenmp", "-shared", "-fPIC"]
# -march of each build and the suffix of its file
ISAS = (("x86-64-v3", ""), ("x86-64-v4", "_v4"))

COMMON_H = """#ifndef COMMON_H
#define COMMON_H
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>
#include <fstream>
#include <iostream>
extern double ref_cfl, ref_gamma, ref_tau_scale, ref_tmax;
extern std::string ref_datain, ref_dataout;
#define REAL    double
#define DATAIN  ref_datain
#define DATAOUT ref_dataout
#define PI     3.14159265358979323846
#define TDIGIT 7
#define N      {N}
#define NP     {NP}
#define NFP    {NFP}
#define NFACE  4
#define NROT   3
#define NVAR   {NVAR}
#define TMAX   ref_tmax
#define CFL    ref_cfl
#define GAMMA  ref_gamma
#define TAU_SCALE ref_tau_scale
#include "{REF}/utils/src/cpp/io.cpp"
#include "{REF}/dim3/src/cpp/{P}_data.cpp"
#include "{REF}/dim3/src/cpp/{P}_dglm.cpp"
#include "{REF}/dim3/src/cpp/{P}_time.cpp"
#endif
"""


# common.h of the reference GPU path (the launcher's macros for one
# configuration, dglm_3d_launcher.py:410-456): CFL, GAMMA, TAU_SCALE and TMAX
# are compile-time here because the device kernels read GAMMA and TAU_SCALE
GPU_COMMON_H = """#ifndef COMMON_H
#define COMMON_H
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>
#include <fstream>
#include <iostream>
#include <cuda_runtime.h>
#include <cublas_v2.h>
extern std::string ref_datain, ref_dataout;
#define REAL    double
#define DATAIN  ref_datain
#define DATAOUT ref_dataout
#define PI     3.14159265358979323846
#define TDIGIT 7
#define N      {N}
#define NP     {NP}
#define NFP    {NFP}
#define NFACE  4
#define NROT   3
#define NVAR   5
#define TMAX   {TMAX}
#define CFL    {CFL}
#define GAMMA  {GAMMA}
#define TAU_SCALE {TAU}
#define FMAX fmax
#define cudaSharedMemBankSizeTByte cudaSharedMemBankSizeEightByte
#define cublasITAMAX cublasIdamax
#define cublasTGEMM cublasDgemm
#define cublasTGEMMBatched cublasDgemmBatched
#define DEVID  -1
#define TPB    256
#define TPBV   {TPBV}
#define pNP    {PNP}
#define pNFF   {PNFF}
#include "{REF}/utils/src/cpp/io.cpp"
#include "{REF}/dim3/src/cuda/euler_nopad_data_host.cu"
#include "{REF}/dim3/src/cuda/euler_nopad_data_dev.cu"
#include "{REF}/dim3/src/cuda/euler_nopad_dglm.cu"
#include "{REF}/dim3/src/cuda/euler_nopad_time.cu"
#endif
"""


def _tpb_maxv(nff):
    """The launcher's block size for calc_maxv (dglm_3d_launcher.py:414-429):
    the even multiple of NFF closest to 256, 512 or 1024."""
    best, diff = -1, 1024
    m = 2
    while nff * m <= 1024:
        for ref in (256, 512, 1024):
            if abs(nff * m - ref) < diff:
                diff, best = abs(nff * m - ref), nff * m
        m += 2
    return best


def build_gpu_solver(N=4, cfl=0.4, gamma=1.4, tau_scale=1.2, tmax=1000.0, force=False):
    """The reference Euler GPU path (CUDA + cuBLAS) for one configuration,
    compiled for sm_100a as the launcher compiles it (nvcc -O3 -std=c++11
    -lcublas, dglm_3d_launcher.py:459) into _ref/libref_gpu_euler_N{N}.so,
    with oracle/ref_gpu_driver.cu around its runRK.  DEVID -1: the calling
    process's current device."""
    Np = (N + 1) * (N + 2) * (N + 3) // 6
    Nfp = (N + 1) * (N + 2) // 2
    bdir = os.path.join(OUT, f"build_gpu_euler_N{N}")
    os.makedirs(bdir, exist_ok=True)
    so = os.path.join(OUT, f"libref_gpu_euler_N{N}.so")
    drv = os.path.join(HERE, "ref_gpu_driver.cu")
    if not force and os.path.exists(so) and os.path.getmtime(so) > os.path.getmtime(drv):
        return so
    pad = lambda x: ((x - 1) // 32 + 1) * 32
    with open(os.path.join(bdir, "common.h"), "w") as f:
        f.write(GPU_COMMON_H.format(N=N, NP=Np, NFP=Nfp, TMAX=repr(float(tmax)),
                                    CFL=repr(float(cfl)), GAMMA=repr(float(gamma)),
                                    TAU=repr(float(tau_scale)), TPBV=_tpb_maxv(4 * Nfp),
                                    PNP=pad(Np), PNFF=pad(4 * Nfp), REF=REF))
    _run(["nvcc", "-O3", "-std=c++11", "-gencode", "arch=compute_100a,code=sm_100a",
          "-shared", "-Xcompiler", "-fPIC", "-I", bdir, drv, "-o", so, "-lcublas"])
    return so


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(" ".join(cmd) + "\n" + r.stdout)


def build_solver(phys: str, N: int, force=False) -> str:
    Np = (N + 1) * (N + 2) * (N + 3) // 6
    Nfp = (N + 1) * (N + 2) // 2
    nvar = 5 if phys == "euler" else 1
    bdir = os.path.join(OUT, f"build_{phys}_N{N}")
    os.makedirs(bdir, exist_ok=True)
    drv = os.path.join(HERE, "ref_driver.cpp")
    with open(os.path.join(bdir, "common.h"), "w") as f:
        f.write(COMMON_H.format(N=N, NP=Np, NFP=Nfp, NVAR=nvar, REF=REF, P=phys))
    flag = "-DREF_EULER" if phys == "euler" else "-DREF_ADVEC"
    out = None
    for march, suffix in ISAS:
        so = os.path.join(OUT, f"libref_{phys}_N{N}{suffix}.so")
        if force or not os.path.exists(so) or os.path.getmtime(so) <= os.path.getmtime(drv):
            _run(["g++", *CXXFLAGS, f"-march={march}", flag, "-I", bdir, drv, "-o", so])
        out = out or so
    return out


def build_mesh_cores() -> None:
    import pybind11
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    inc = ["-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"]]
    for name, src in (("mesh_3d_cpp", "mesh_3d_core.cpp"),
                      ("uniform_3d_single_cpp", "uniform_3d_single_core.cpp")):
        out = os.path.join(OUT, name + suffix)
        if os.path.exists(out):
            continue
        _run(["g++", "-O3", "-shared", "-std=c++17", "-fPIC", *inc,
              os.path.join(REF, "dim3/src/cpp", src), "-o", out])


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--orders", default="1-6")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-mesh", action="store_true")
    a = ap.parse_args(argv)
    if not os.path.isdir(os.path.join(REF, "dim3/src/cpp")):
        print(f"reference tree not found at {REF}; oracle/_ref not built")
        return 0
    lo, _, hi = a.orders.partition("-")
    orders = range(int(lo), int(hi or lo) + 1)
    os.makedirs(OUT, exist_ok=True)
    for phys in ("euler", "advec"):
        for N in orders:
            build_solver(phys, N, force=a.force)
    try:
        build_gpu_solver(4)
    except Exception as e:              # nvcc or cuBLAS missing: CPU baselines only
        print("reference GPU path not built:", e)
    if not a.no_mesh:
        try:
            build_mesh_cores()
        except Exception as e:          # pybind11 headers missing: fixtures only
            print("mesh cores not built:", e)
    print("oracle/_ref built:", sorted(os.listdir(OUT)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
