"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference tree is mounted (it is not on the GPU machines):

    python oracle/build_ref.py          # compiles the reference into oracle/_ref
    python tests/golden/make_golden.py

Fixtures (numpy .npz, committed):

* refelem.npz  -- the reference's stored operator matrices (dim3/data/
                  bin_mats/N{n}/*.bin): full for N <= 4, seeded samples and
                  norms for N = 5, 6; Fmask/FmaskP from the reference's
                  FaceMask (operator_3d_face.py:74-123) for N = 1..6.
* mesh.npz     -- the reference Mesh3D (mesh_3d.py, with its C++ cores
                  rebuilt from dim3/src/cpp) on a periodic 3^3-hex mesh at
                  N = 3 and a mixed periodic/boundary 3x2x3 mesh at N = 2.
* kernels.npz  -- the reference CPU solver (oracle/_ref) run on this
                  package's inputs: every intermediate of one right-hand side
                  (maxv, tau, ub, fluxLM, fluxR/S/T, utmp) and the state and
                  dt after 10 steps, for advection N=3 and Euler N=3 on the
                  2^3-hex periodic mesh (K = 48).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# the reference tree: $DGLM_REFERENCE_ROOT, else a "reference" directory
# beside the repository
REF = os.environ.get("DGLM_REFERENCE_ROOT",
                     os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(
                         os.path.dirname(os.path.abspath(__file__))))), "reference"))
sys.path.insert(0, ROOT)


def refelem():
    sys.path.insert(0, os.path.join(REF, "dim3/src/python"))
    from operator_3d_face import FaceMask
    out = {}
    rng = np.random.default_rng(20240601)
    for N in range(1, 7):
        Np = (N + 1) * (N + 2) * (N + 3) // 6
        Nfp = (N + 1) * (N + 2) // 2
        d = os.path.join(REF, "dim3/data/bin_mats", f"N{N}")
        shapes = {"rst": (Np, 3), "WDr": (Np, Np), "WDs": (Np, Np), "WDt": (Np, Np),
                  "LIFT": (Np, 4 * Nfp), "M": (Np, Np), "Emat": (Np, 4 * Nfp)}
        for name, shp in shapes.items():
            a = np.fromfile(os.path.join(d, name + ".bin")).reshape(shp)
            if N <= 4:
                out[f"N{N}_{name}"] = a
            else:
                idx = rng.choice(a.size, size=min(256, a.size), replace=False)
                out[f"N{N}_{name}_idx"] = idx
                out[f"N{N}_{name}_val"] = a.ravel()[idx]
                out[f"N{N}_{name}_fro"] = np.linalg.norm(a)

        class T:
            pass
        t = T()
        t.N, t.Nface, t.Nrot, t.Nfp = N, 4, 3, Nfp
        t.rst = np.fromfile(os.path.join(d, "rst.bin")).reshape(Np, 3)
        Fm, FmP = FaceMask(t).make_face_mask()
        out[f"N{N}_Fmask"], out[f"N{N}_FmaskP"] = Fm, FmP
    np.savez_compressed(os.path.join(HERE, "refelem.npz"), **out)


def mesh():
    sys.path.insert(0, os.path.join(REF, "dim3/src/python"))
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))   # rebuilt cores first
    from tetra import TetraRef
    from operator_3d_ref import Operator3DRef
    from operator_3d_face import Operator3DFace
    from uniform_3d_single import Uniform3DSingle
    from mesh_3d import Mesh3D
    import mesh_3d_cpp
    assert os.path.dirname(mesh_3d_cpp.__file__).endswith("_ref"), mesh_3d_cpp.__file__
    out = {}
    cases = {"pbc": (3, (4, 4, 4), {"x": "pbc", "y": "pbc", "z": "pbc"}),
             "mixed": (2, (4, 3, 4), {"x": "bc1", "y": "pbc", "z": "bc2"})}
    for tag, (N, (nx, ny, nz), bc) in cases.items():
        tet = TetraRef(N, 2)
        opf = Operator3DFace(Operator3DRef(tet))
        m = Mesh3D(opf, Uniform3DSingle(nx, ny, nz, 0, 1, 0, 1, 0, 1, bc))
        for name in ("EtoV", "EtoE", "EtoB", "vmapM", "vmapP", "vmapF", "PX", "PY", "PZ",
                     "J", "rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz", "NX", "NY",
                     "NZ", "sJ", "Fscale"):
            out[f"{tag}_{name}"] = getattr(m, name)
        out[f"{tag}_N"], out[f"{tag}_dims"] = N, np.array([nx, ny, nz])
    np.savez_compressed(os.path.join(HERE, "mesh.npz"), **out)


def kernels():
    import oracle
    from exadglm_b200 import problem as P
    out = {}
    cases = {"advec": P.advection_gaussian(n=2, N=3, width2=0.05),
             "euler": P.euler_sine(n=2, N=3, noise=1e-3, seed=7)}
    for tag, p in cases.items():
        r = oracle.RefSolver(p)
        rhs = r.rhs()
        for k in ("maxv", "tau", "ub", "fluxLM", "fluxR", "fluxS", "fluxT", "utmp"):
            out[f"{tag}_{k}"] = rhs[k]
        out[f"{tag}_dt0"] = rhs["dt"]
        r.set_state(p.u0)
        dts = []
        for _ in range(10):
            r.run(1)
            dts.append(r.time()[1])
        out[f"{tag}_u10"] = r.get_state()
        out[f"{tag}_dt10"] = np.array(dts)
        out[f"{tag}_t10"] = r.time()[0]
        r.close()
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), **out)


if __name__ == "__main__":
    refelem()
    mesh()
    kernels()
    for f in ("refelem.npz", "mesh.npz", "kernels.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)) // 1024, "KB")
