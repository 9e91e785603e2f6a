"""Reference-element operators against the reference's stored matrices
(tests/golden/refelem.npz, made by tests/golden/make_golden.py from
dim3/data/bin_mats) and against the properties the reference's own tests
check (dim3/tests/test_operator_3d_ref.py, test_operator_3d_face.py,
test_jacobi.py)."""
import os

import numpy as np
import pytest

from exadglm_b200.refelem import dims, gll_nodes, jacobi_p, ref_element

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "refelem.npz"))
# the reference stores float64 roundings of 21-digit mpmath results; ours come
# from 64-bit-mantissa arithmetic: agreement to a few ulp of the largest entry
TOL = 4e-15


def rel_max(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("N", [1, 2, 3, 4])
@pytest.mark.parametrize("name", ["rst", "WDr", "WDs", "WDt", "LIFT", "M", "Emat"])
def test_full_matrices_match_reference(N, name):
    re = ref_element(N)
    assert rel_max(getattr(re, name), GOLD[f"N{N}_{name}"]) < TOL


@pytest.mark.parametrize("N", [5, 6])
@pytest.mark.parametrize("name", ["rst", "WDr", "WDs", "WDt", "LIFT", "M", "Emat"])
def test_sampled_matrices_match_reference(N, name):
    a = getattr(ref_element(N), name)
    vals = GOLD[f"N{N}_{name}_val"]
    np.testing.assert_allclose(a.ravel()[GOLD[f"N{N}_{name}_idx"]], vals,
                               rtol=0, atol=TOL * np.abs(a).max())
    assert abs(np.linalg.norm(a) - GOLD[f"N{N}_{name}_fro"]) < 1e-13 * GOLD[f"N{N}_{name}_fro"]


@pytest.mark.parametrize("N", range(1, 7))
def test_face_masks_identical(N):
    re = ref_element(N)
    np.testing.assert_array_equal(re.Fmask, GOLD[f"N{N}_Fmask"])
    np.testing.assert_array_equal(re.FmaskP, GOLD[f"N{N}_FmaskP"])


def test_face_mask_n3_literal():
    """The N=3 Fmask/FmaskP vectors pinned as literals by the reference's
    dim3/tests/test_operator_3d_face.py (test_make_face_mask)."""
    re = ref_element(3)
    fm = [[3, 2, 1, 0, 6, 5, 4, 8, 7, 9], [0, 1, 2, 3, 10, 11, 12, 16, 17, 19],
          [3, 6, 8, 9, 12, 14, 15, 17, 18, 19], [9, 7, 4, 0, 15, 13, 10, 18, 16, 19]]
    fmp = [[[0, 1, 2, 3, 4, 5, 6, 7, 8, 9], [3, 6, 8, 9, 2, 5, 7, 1, 4, 0],
            [9, 7, 4, 0, 8, 5, 1, 6, 2, 3]],
           [[3, 2, 1, 0, 12, 11, 10, 17, 16, 19], [0, 10, 16, 19, 1, 11, 17, 2, 12, 3],
            [19, 17, 12, 3, 16, 11, 2, 10, 1, 0]],
           [[9, 8, 6, 3, 15, 14, 12, 18, 17, 19], [3, 12, 17, 19, 6, 14, 18, 8, 15, 9],
            [19, 18, 15, 9, 17, 14, 8, 12, 6, 3]],
           [[0, 4, 7, 9, 10, 13, 15, 16, 18, 19], [9, 15, 18, 19, 7, 13, 16, 4, 10, 0],
            [19, 16, 10, 0, 18, 13, 4, 15, 7, 9]]]
    np.testing.assert_array_equal(re.Fmask, fm)
    np.testing.assert_array_equal(re.FmaskP, fmp)


@pytest.mark.parametrize("N", [2, 3, 5])
def test_emat_sums_to_total_face_area(N):
    # sum over faces of the reference-face areas: 3 faces of area 2 and the
    # slanted one of area 2*sqrt(3), in face-Jacobian units -> 8 as in the
    # reference's test (sum(Emat) = 8)
    assert ref_element(N).Emat.sum() == pytest.approx(8.0, rel=1e-13)


@pytest.mark.parametrize("N", [1, 3, 6])
def test_mass_matrix_integrates_volume(N):
    # the reference tetrahedron has volume 4/3
    assert ref_element(N).M.sum() == pytest.approx(4.0 / 3.0, rel=1e-13)


@pytest.mark.parametrize("N", [2, 4])
def test_derivative_exact_on_polynomials(N):
    re = ref_element(N)
    r, s, t = re.rst[:, 0], re.rst[:, 1], re.rst[:, 2]
    f = r ** N + s * t ** (N - 1) + r * s
    np.testing.assert_allclose(re.Dr @ f, N * r ** (N - 1) + s, atol=1e-11)
    np.testing.assert_allclose(re.Dt @ f, (N - 1) * s * t ** (N - 2), atol=1e-11)


# known-answer values of the reference's dim3/tests/test_jacobi.py
_GLL = {3: [-1, -0.447213595499958, 0.4472135954999580, 1],
        4: [-1, -0.654653670707977, 0, 0.654653670707977, 1],
        5: [-1, -0.765055323929465, -0.285231516480645, 0.285231516480645, 0.765055323929465, 1]}
_JAC = {2: ([1.581138830084190, -0.790569415042095, 1.581138830084190],
            [-4.743416490252569, 0, 4.743416490252569]),
        3: ([-1.87082869338697, 0.836660026534076, -0.836660026534076, 1.87082869338697],
            [11.224972160321824, 0, 0, 11.224972160321824]),
        4: ([2.121320343559642, -0.909137290096990, 0.795495128834866, -0.909137290096990,
             2.121320343559642], [-21.213203435596430, 0, 0, 0, 21.213203435596430]),
        5: ([-2.345207879911714, 0.984276557099483, -0.812914072195837, 0.812914072195837,
             -0.984276557099483, 2.345207879911714],
            [35.178118198675726, 0, 0, 0, 0, 35.178118198675726])}


@pytest.mark.parametrize("N", [3, 4, 5])
def test_gll_nodes_known_values(N):
    np.testing.assert_allclose(gll_nodes(N).astype(float), _GLL[N], atol=1e-14)


@pytest.mark.parametrize("N", [2, 3, 4, 5])
def test_jacobi_known_values(N):
    from exadglm_b200.refelem import grad_jacobi_p
    r = gll_nodes(N)
    j, dp = _JAC[N]
    np.testing.assert_allclose(jacobi_p(r, 0, 0, N).astype(float), j, atol=1e-13)
    np.testing.assert_allclose(grad_jacobi_p(r, 0, 0, N).astype(float), dp, atol=1e-12)


def test_dims():
    assert dims(4) == (35, 15) and dims(6) == (84, 28)
