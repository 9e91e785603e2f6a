"""Compact face maps on the host (dglm_compact_face_maps): the form the
device kernels read when Solver.set_compact_face_maps is on.  Round trip to
vmapP on the benchmark meshes, agreement with the Python compaction of
mesh.compact_face_maps, and the refusals."""
import numpy as np
import pytest

from exadglm_b200 import capi
from exadglm_b200 import problem as P


def expand(etoe, code, lists, Np):
    return etoe[:, :, None] * Np + lists[code]


@pytest.mark.parametrize("phys,N,n", [("euler", 4, 3), ("euler", 4, 16), ("euler", 6, 4),
                                      ("advection", 3, 5), ("euler", 1, 3), ("euler", 8, 2)])
def test_round_trip(phys, N, n):
    prob = (P.euler_sine(n=n, N=N) if phys == "euler"
            else P.advection_gaussian(n=n, N=N, width2=0.05))
    vm = prob.datain_arrays()["vmapP"].reshape(prob.K, 4, -1)
    Nfp = vm.shape[2]
    etoe, code, lists = capi.compact_face_maps(vm, prob.Np, Nfp)
    assert np.array_equal(expand(etoe, code, lists, prob.Np), vm)
    # a conforming tetrahedral mesh: one list per (neighbour face, orientation)
    assert 1 <= len(lists) <= 24
    # every list is a face of the reference element, in some node order
    Fm = prob.datain_arrays()["Fmask"].reshape(4, Nfp)
    faces = [set(f.tolist()) for f in Fm]
    assert all(set(l.tolist()) in faces for l in lists)
    # 5 bytes per face against 4 Nfp
    assert etoe.nbytes + code.nbytes == 20 * prob.K


@pytest.mark.parametrize("N", [2, 4])
@pytest.mark.parametrize("bc", [{"x": "pbc", "y": "pbc", "z": "pbc"},
                                {"x": "bc1", "y": "pbc", "z": "bc2"}])
def test_agrees_with_python_compaction(N, bc):
    """Same neighbours as mesh.compact_face_maps, on periodic faces and on
    boundary faces that map onto themselves; one code per (EtoF, EtoR)."""
    from exadglm_b200.mesh import Mesh3D, UniformBox, compact_face_maps
    m = Mesh3D(N, UniformBox(4, 3, 3, bc=bc), high_order=False)
    etoe, code, lists = capi.compact_face_maps(m.vmapP, m.Np, m.Nfp)
    vm = np.asarray(m.vmapP).reshape(-1, 4, m.Nfp)
    assert np.array_equal(expand(etoe, code, lists, m.Np), vm)
    E2, F2, R2 = compact_face_maps(m.vmapP, m.ref, m.Np)
    assert np.array_equal(E2, etoe)
    key = F2.astype(np.int64) * 8 + R2
    for k in np.unique(key):
        assert len(np.unique(code[key == k])) == 1


def test_refusals():
    prob = P.euler_sine(n=3, N=4)
    vm = np.array(prob.datain_arrays()["vmapP"], copy=True).reshape(prob.K, 4, -1)
    bad = vm.copy()
    bad[0, 0, 0] = ((int(bad[0, 0, 1]) // prob.Np + 1) % prob.K) * prob.Np
    with pytest.raises(capi.DglmError, match="spans several elements"):
        capi.compact_face_maps(bad, prob.Np, prob.Nfp)
    with pytest.raises(capi.DglmError, match="max_lists"):
        capi.compact_face_maps(vm, prob.Np, prob.Nfp, max_lists=2)
    neg = vm.copy()
    neg[3, 2, 0] = -1
    with pytest.raises(capi.DglmError, match="outside"):
        capi.compact_face_maps(neg, prob.Np, prob.Nfp)
