"""Compact face maps (dglm_set_compact_face_maps) on the GPU.

With the maps on, the producer warps of the persistent stage kernels form
each neighbour node index as EtoE Np + list[code][j] instead of reading
vmapP; the gathered values are the same, so a run must equal the vmapP run
bit for bit, for every kernel family that reads them (FP64 pipelined,
tensor-memory TF32 and BF16, one and two accumulators) and for advection.
A face whose trace spans two elements is refused."""
import numpy as np
import pytest

from exadglm_b200 import problem as P
from exadglm_b200.capi import DglmError, Solver, variants

pytestmark = pytest.mark.gpu

STEPS = 5


def make(phys, N):
    if phys == "euler":
        return P.euler_sine(n=3, N=N, noise=1e-3, seed=3)
    return P.advection_gaussian(n=3, N=N, width2=0.05)


@pytest.mark.parametrize("phys,N,prec", [
    ("euler", 4, "fp64"), ("euler", 5, "fp64"), ("advection", 4, "fp64"),
    ("euler", 4, "tf32x3"), ("euler", 4, "bf16x3"), ("euler", 6, "bf16x3"),
])
def test_compact_maps_equal_vmapP(phys, N, prec):
    prob = make(phys, N)
    ref = Solver(prob, precision=prec)
    desc = variants(phys, N)[ref.variant()]
    ref.step(STEPS)
    u_ref = ref.get_state()
    ref.close()
    s = Solver(prob, precision=prec)
    s.set_compact_face_maps(True)
    lists = s.face_map_lists()
    # a conforming tetrahedral mesh: one list per (neighbour face, orientation)
    assert 1 <= lists <= 24, lists
    s.step(STEPS)
    u = s.get_state()
    print(f"{phys} N={N} {prec} {desc}: {lists} node lists, "
          f"max |diff| {np.max(np.abs(u - u_ref)):.1e}")
    assert np.array_equal(u, u_ref), desc
    # and back to vmapP on the same handle
    s.set_compact_face_maps(False)
    s.set_state(prob.u0)
    s.step(STEPS)
    assert np.array_equal(s.get_state(), u_ref)
    s.close()


def test_compact_maps_refuse_a_split_face():
    prob = make("euler", 4)
    arr = {k: np.array(v, copy=True) for k, v in prob.datain_arrays().items()}
    vm = arr["vmapP"].reshape(-1)
    # face point 0 of element 0 moved to another element than the rest of its face
    other = (int(vm[1]) // prob.Np + 1) % prob.K
    vm[0] = other * prob.Np
    s = Solver(prob, arrays=arr)
    with pytest.raises(DglmError, match="spans several elements"):
        s.set_compact_face_maps(True)
    assert s.face_map_lists() == 0
    s.close()
