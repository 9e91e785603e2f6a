"""Mesh arrays against the reference Mesh3D (tests/golden/mesh.npz, made from
the reference's own mesh code with its C++ cores rebuilt from source) and
the geometric properties its tests check (dim3/tests/test_uniform_3d_single.py,
test_mesh_3d_common.py, test_mesh_3d_serial_uniform_pbc.py)."""
import os

import numpy as np
import pytest

from exadglm_b200.mesh import Mesh3D, UniformBox, uniform_mesh

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "mesh.npz"))
CASES = {"pbc": {"x": "pbc", "y": "pbc", "z": "pbc"},
         "mixed": {"x": "bc1", "y": "pbc", "z": "bc2"}}


def build(tag):
    nx, ny, nz = (int(v) for v in GOLD[f"{tag}_dims"])
    return Mesh3D(int(GOLD[f"{tag}_N"]), UniformBox(nx, ny, nz, bc=CASES[tag]))


@pytest.mark.parametrize("tag", ["pbc", "mixed"])
def test_index_arrays_identical(tag):
    m = build(tag)
    for name in ("EtoV", "vmapM", "vmapP", "vmapF", "EtoB"):
        np.testing.assert_array_equal(getattr(m, name), GOLD[f"{tag}_{name}"], err_msg=name)
    # EtoE agrees wherever the reference has a neighbour
    ref = GOLD[f"{tag}_EtoE"]
    np.testing.assert_array_equal(m.EtoE[ref >= 0], ref[ref >= 0])


@pytest.mark.parametrize("tag", ["pbc", "mixed"])
def test_geometry_matches(tag):
    m = build(tag)
    for name in ("PX", "PY", "PZ", "J", "rx", "ry", "rz", "sx", "sy", "sz", "tx", "ty", "tz",
                 "NX", "NY", "NZ", "sJ", "Fscale"):
        np.testing.assert_allclose(getattr(m, name), GOLD[f"{tag}_{name}"], rtol=0,
                                   atol=1e-15 * max(1.0, np.abs(GOLD[f"{tag}_{name}"]).max()),
                                   err_msg=name)


@pytest.mark.parametrize("N,n", [(1, 2), (3, 3), (4, 4)])
def test_vmapP_involution_and_coincidence(N, n):
    """vmapP points to a coincident node (mod the period) and is an
    involution on a periodic mesh."""
    m = uniform_mesh(N, n)
    vM, vP = m.vmapM.ravel(), m.vmapP.ravel()
    x = np.stack([m.PX.ravel(), m.PY.ravel(), m.PZ.ravel()], axis=1)
    d = x[vM] - x[vP]
    d -= np.round(d)                      # unit period
    assert np.abs(d).max() < 1e-12
    # per face pair: if node j of face (e,f) maps to position j' of the
    # neighbour face (e',f'), then j' maps back to j
    K, Nfp = m.Nelem, m.Nfp
    VM, VP = m.vmapM.reshape(K * 4, Nfp), m.vmapP.reshape(K * 4, Nfp)
    nb = m.vmapF.ravel()
    pos = np.argmax(VM[nb][:, None, :] == VP[:, :, None], axis=2)   # (4K, Nfp) -> j'
    back = VP[nb][np.arange(4 * K)[:, None], pos]
    np.testing.assert_array_equal(back, VM)
    F = m.vmapF.ravel()
    np.testing.assert_array_equal(F[F], np.arange(F.size))


def test_volume_and_normals():
    m = uniform_mesh(3, 3)
    assert (m.J * 4.0 / 3.0).sum() == pytest.approx(1.0, rel=1e-14)   # unit cube
    n = np.stack([m.NX, m.NY, m.NZ], axis=-1)
    np.testing.assert_allclose(np.linalg.norm(n, axis=-1), 1.0, rtol=1e-15)
    # neighbouring faces have opposite normals
    F = m.vmapF.ravel()
    nf = n.reshape(-1, 3)
    np.testing.assert_allclose(nf + nf[F], 0.0, atol=1e-14)


@pytest.mark.parametrize("N,n", [(3, 3), (4, 2)])
def test_face_jacobian_matches_triangle_areas(N, n):
    """2 sJ is the physical area of a face (the reference face has area 2 in
    the face parametrisation, sum(Emat) = 8 over 4 faces), with sJ = Fscale J.
    Summed over all faces it equals the summed surface areas of the tets
    computed from their vertices (test_mesh_3d_common.py's sJ check, in a
    form independent of the face numbering)."""
    m = uniform_mesh(N, n)
    sJ = m.Fscale * m.J[:, None]
    V = np.stack([m.VX, m.VY, m.VZ], axis=1)[m.EtoV]             # (K, 4, 3)
    area = 0.0
    for tri in ((0, 1, 2), (0, 1, 3), (1, 2, 3), (0, 2, 3)):
        a, b, c = V[:, tri[0]], V[:, tri[1]], V[:, tri[2]]
        area += 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum()
    assert (2.0 * sJ).sum() == pytest.approx(area, rel=1e-13)
    assert np.all(sJ > 0)


@pytest.mark.parametrize("N,n", [(3, 3), (5, 2)])
def test_normals_orthogonal_to_their_faces(N, n):
    """n is orthogonal to every chord between two nodes of its face
    (test_mesh_3d_common.py's normal orthogonality)."""
    m = uniform_mesh(N, n)
    X = np.stack([m.PX, m.PY, m.PZ], axis=-1)                      # (K, Np, 3)
    nrm = np.stack([m.NX, m.NY, m.NZ], axis=-1)                    # (K, 4, 3)
    for f in range(4):
        pts = X[:, m.ref.Fmask[f]]                                 # (K, Nfp, 3)
        chords = pts - pts[:, :1]
        dots = np.einsum("kjd,kd->kj", chords, nrm[:, f])
        assert np.abs(dots).max() < 1e-13


def test_element_counts():
    b = UniformBox(7, 7, 7)
    assert b.Nelem == 1296 and b.EtoV.shape == (1296, 4)


def test_rejects_degenerate_periodic_axis():
    with pytest.raises(ValueError):
        UniformBox(2, 4, 4)


def test_l2_error_matches_per_element_loop():
    """The vectorised mass-weighted L2 error (a14) against a loop over the
    elements written as dglm_3d_launcher.py:328-355 computes it:
    sum_e J_e (u_ref - interpM u_num)^T high_M (u_ref - interpM u_num)."""
    from exadglm_b200 import problem as P
    p = P.euler_sine(n=2, N=3)
    ref = p.mesh.ref
    rng = np.random.default_rng(4)
    u_num = rng.standard_normal(p.K * p.Np)
    u_ref = rng.standard_normal(p.K * ref.high_Np)
    total = 0.0
    for e in range(p.K):
        E = u_ref[e * ref.high_Np:(e + 1) * ref.high_Np] - ref.interpM @ u_num[e * p.Np:(e + 1) * p.Np]
        total += p.mesh.J[e] * (E @ ref.high_M @ E)
    assert P.l2_error(p, u_ref, u_num, apply_sqrt=False) == pytest.approx(total, rel=1e-13)
    assert P.l2_error(p, u_ref, u_num) == pytest.approx(np.sqrt(total), rel=1e-13)


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("tag", ["pbc", "mixed"])
def test_compact_face_maps_regenerate_vmapP(N, tag):
    """(EtoE, EtoF, orientation) per face regenerates vmapP exactly, for
    periodic faces and for boundary faces that map onto themselves; 24 bytes
    per element against 16 Nfp."""
    from exadglm_b200.mesh import compact_face_maps, expand_face_maps
    m = Mesh3D(N, UniformBox(4, 3, 3, bc=CASES[tag]), high_order=False)
    EtoE, EtoF, EtoR = compact_face_maps(m.vmapP, m.ref, m.Np)
    np.testing.assert_array_equal(expand_face_maps(EtoE, EtoF, EtoR, m.ref, m.Np), m.vmapP)
    assert EtoE.nbytes + EtoF.nbytes + EtoR.nbytes == 24 * m.Nelem
    inner = m.EtoE >= 0
    np.testing.assert_array_equal(EtoE[inner], m.EtoE[inner])
    np.testing.assert_array_equal(EtoF[inner], m.EtoF[inner])


def test_compact_face_maps_reject_broken_maps():
    from exadglm_b200.mesh import compact_face_maps
    m = uniform_mesh(3, 2)
    bad = m.vmapP.copy()
    bad[0, 0, 0] = bad[5, 2, 0]          # one node from another element
    with pytest.raises(ValueError):
        compact_face_maps(bad, m.ref, m.Np)
    bad = m.vmapP.copy()
    bad[0, 0, [1, 2]] = bad[0, 0, [2, 1]]  # not a rotation or reflection
    with pytest.raises(ValueError):
        compact_face_maps(bad, m.ref, m.Np)
