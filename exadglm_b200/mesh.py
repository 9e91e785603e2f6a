"""Uniform tetrahedral box meshes and their DG geometry, vectorised.

Produces exactly the arrays the solver reads from ``datain/`` (the
reference's Mesh3D outputs, dim3/src/python/mesh_3d.py:9-116):

* ``EtoV`` (K,4) and vertex coordinates; each hexahedron is cut into six
  tetrahedra around its main diagonal v0-v7 in the reference's order
  (dim3/src/cpp/uniform_3d_single_core.cpp:8-67) -- the element numbering is
  part of the data format;
* ``PX, PY, PZ`` (K,Np) node coordinates (mesh_3d_core.cpp:10-63);
* affine metrics ``J, rx..tz`` (K,) (mesh_3d_core.cpp:66-145);
* unit normals ``nx, ny, nz``, ``sJ`` and ``Fscale = sJ/J`` (K,4)
  (mesh_3d_core.cpp:237-306);
* ``vmapM, vmapP`` (K,4,Nfp) and ``vmapF`` (K,4) (mesh_3d_core.cpp:309-356),
  ``EtoB`` (K,4) with -99 on interior/periodic faces and the boundary tag
  elsewhere (uniform_3d_single_core.cpp:220-271).

Connectivity is found here by matching face centroids (in integer grid
units, reduced over periodic axes) instead of hand-written neighbour tables,
and the face-node correspondence by matching barycentric coordinates on the
shared face; both give the same arrays as the reference's tables because the
neighbour face of a face, and the neighbour node of a face node, are unique.
"""
from __future__ import annotations

import itertools
import re

import numpy as np

from .refelem import RefElement, ref_element

# local vertex triples of the four faces: 0 t=-1, 1 s=-1, 2 r+s+t=-1, 3 r=-1
# (operator_3d_face.py:84-88)
FACE_VERTS = np.array([[1, 0, 2], [0, 1, 3], [1, 2, 3], [2, 0, 3]], np.int64)

# six tetrahedra per hexahedron, as local hex corners (0..7, bit order z,y,x)
HEX_TETS = np.array([[0, 7, 3, 1], [0, 7, 2, 3], [0, 7, 6, 2],
                     [0, 7, 4, 6], [0, 7, 5, 4], [0, 7, 1, 5]], np.int64)


def _parse_bc(spec):
    if spec == "pbc":
        return -1
    m = re.findall(r"bc(\d+)", spec)
    if not m:
        raise ValueError(f"boundary spec {spec!r} is neither 'pbc' nor 'bc<tag>'")
    return int(m[0])


class UniformBox:
    """``nx*ny*nz`` grid points, ``(nx-1)(ny-1)(nz-1)`` hexahedra, six
    tetrahedra each (the reference's Uniform3DSingle, uniform_3d_single.py:8).

    ``bc`` maps each axis to 'pbc' (periodic) or 'bc<tag>'.
    """

    def __init__(self, nx, ny, nz, x1=0.0, x2=1.0, y1=0.0, y2=1.0, z1=0.0, z2=1.0,
                 bc=None):
        bc = bc or {"x": "pbc", "y": "pbc", "z": "pbc"}
        self.nx, self.ny, self.nz = nx, ny, nz
        self.lo = np.array([x1, y1, z1], np.float64)
        self.hi = np.array([x2, y2, z2], np.float64)
        self.tags = np.array([_parse_bc(bc["x"]), _parse_bc(bc["y"]), _parse_bc(bc["z"])])
        for n, tag in zip((nx, ny, nz), self.tags):
            if n < 2:
                raise ValueError("need at least 2 grid points per axis")
            if tag < 0 and n < 3:
                raise ValueError("a periodic axis needs at least 2 cells")
        self.Ncube = (nx - 1) * (ny - 1) * (nz - 1)
        self.Nelem = 6 * self.Ncube
        x = np.linspace(x1, x2, nx)
        y = np.linspace(y1, y2, ny)
        z = np.linspace(z1, z2, nz)
        X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
        self.VXYZ = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
        i, j, k = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1),
                              indexing="ij")
        i, j, k = i.ravel(), j.ravel(), k.ravel()
        corner = np.empty((self.Ncube, 8), np.int64)
        for c in range(8):
            di, dj, dk = (c >> 2) & 1, (c >> 1) & 1, c & 1
            corner[:, c] = ((i + di) * ny + (j + dj)) * nz + (k + dk)
        self.EtoV = corner[:, HEX_TETS].reshape(self.Nelem, 4).astype(np.int32)
        # periodic identification of grid points
        gi, gj, gk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        if self.tags[0] < 0:
            gi = gi % (nx - 1)
        if self.tags[1] < 0:
            gj = gj % (ny - 1)
        if self.tags[2] < 0:
            gk = gk % (nz - 1)
        self.vertex_class = ((gi * ny + gj) * nz + gk).ravel()
        self.EtoE, self.EtoF, self.EtoB = self._connect()

    def _connect(self):
        K = self.Nelem
        nx, ny, nz = self.nx, self.ny, self.nz
        gi, gj, gk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        grid = np.stack([gi.ravel(), gj.ravel(), gk.ravel()], axis=1)       # (Nv,3)
        # 3 x face centroid in grid units, reduced over periodic axes: two
        # faces coincide exactly when these integer triples are equal
        c3 = grid[self.EtoV.astype(np.int64)[:, FACE_VERTS]].sum(axis=2)   # (K,4,3)
        span = []
        for ax, n in enumerate((nx, ny, nz)):
            if self.tags[ax] < 0:
                c3[..., ax] %= 3 * (n - 1)
            span.append(3 * (n - 1) + 1)
        key = ((c3[..., 0] * span[1]) + c3[..., 1]) * span[2] + c3[..., 2]
        key = key.ravel()
        order = np.argsort(key, kind="stable")
        ks = key[order]
        EtoE = np.full(4 * K, -99, np.int64)
        EtoF = np.zeros(4 * K, np.int64)
        same = ks[1:] == ks[:-1]
        if np.any(same[1:] & same[:-1]):
            raise ValueError("a face is shared by more than two elements")
        a, b = order[:-1][same], order[1:][same]
        EtoE[a], EtoF[a] = b // 4, b % 4
        EtoE[b], EtoF[b] = a // 4, a % 4
        bnd = EtoE < 0
        EtoF[bnd] = np.arange(4 * K)[bnd] % 4
        EtoB = np.full(4 * K, -99, np.int64)
        if np.any(bnd):
            # a boundary face lies on the plane of one non-periodic axis
            cent = self.VXYZ[self.EtoV.astype(np.int64)[:, FACE_VERTS]].mean(axis=2).reshape(-1, 3)
            h = (self.hi - self.lo) / (np.array([self.nx, self.ny, self.nz]) - 1)
            for ax in range(3):
                on = bnd & ((np.abs(cent[:, ax] - self.lo[ax]) < 1e-9 * h[ax]) |
                            (np.abs(cent[:, ax] - self.hi[ax]) < 1e-9 * h[ax]))
                EtoB[on] = self.tags[ax]
            if np.any(EtoB[bnd] < 0):
                raise ValueError("unmatched interior face")
        return (EtoE.reshape(K, 4).astype(np.int32), EtoF.reshape(K, 4).astype(np.int32),
                EtoB.reshape(K, 4).astype(np.int32))


def _face_node_perm(ref: RefElement):
    """T[f, g, p] = positions j' on face g matching the nodes j of face f when
    the face's vertex triple appears in the neighbour under permutation p."""
    Nfp = ref.Nfp
    r, s, t = ref.rst[:, 0], ref.rst[:, 1], ref.rst[:, 2]
    lam = np.stack([-(1 + r + s + t) / 2, (1 + r) / 2, (1 + s) / 2, (1 + t) / 2], axis=1)
    perms = list(itertools.permutations(range(3)))
    T = np.zeros((4, 4, 6, Nfp), np.int64)
    for f in range(4):
        lf = lam[ref.Fmask[f]][:, FACE_VERTS[f]]                     # (Nfp,3)
        for g in range(4):
            lg = lam[ref.Fmask[g]][:, FACE_VERTS[g]]
            for p, pi in enumerate(perms):
                # neighbour vertex pi[k] is this face's vertex k
                d = np.abs(lf[:, None, :] - lg[None, :, list(pi)]).max(axis=2)
                j2 = d.argmin(axis=1)
                if d[np.arange(Nfp), j2].max() > 1e-9:
                    raise AssertionError("face nodes do not match under a vertex permutation")
                T[f, g, p] = j2
    return T, perms


class Mesh3D:
    """DG geometry of a tetrahedral mesh for order N: the arrays of the
    reference's Mesh3D (mesh_3d.py:9-116), computed with numpy.

    ``box`` is a :class:`UniformBox` (or any object with ``VXYZ``, ``EtoV``,
    ``EtoE``, ``EtoF``, ``EtoB`` and ``vertex_class``).
    """

    def __init__(self, N, box, interpN=2, high_order=True):
        ref = ref_element(N, interpN)
        self.ref = self.tet = ref
        self.box = box
        self.N, self.Np, self.Nfp, self.Nface = N, ref.Np, ref.Nfp, 4
        self.Nelem = K = box.Nelem
        V = box.VXYZ
        EtoV = box.EtoV.astype(np.int64)
        self.VX, self.VY, self.VZ = V[:, 0], V[:, 1], V[:, 2]
        self.EtoV, self.EtoE, self.EtoF, self.EtoB = box.EtoV, box.EtoE, box.EtoF, box.EtoB
        v = [V[EtoV[:, q]] for q in range(4)]                       # 4 x (K,3)
        self.PX, self.PY, self.PZ = self._points(v, ref.rst)
        # affine metrics (mesh_3d_core.cpp:66-145 / book GeometricFactors3D)
        xr, xs, xt = [0.5 * (v[q][:, 0] - v[0][:, 0]) for q in (1, 2, 3)]
        yr, ys, yt = [0.5 * (v[q][:, 1] - v[0][:, 1]) for q in (1, 2, 3)]
        zr, zs, zt = [0.5 * (v[q][:, 2] - v[0][:, 2]) for q in (1, 2, 3)]
        J = xr * (ys * zt - zs * yt) - yr * (xs * zt - zs * xt) + zr * (xs * yt - ys * xt)
        self.J = J
        self.rx = (ys * zt - zs * yt) / J
        self.ry = -(xs * zt - zs * xt) / J
        self.rz = (xs * yt - ys * xt) / J
        self.sx = -(yr * zt - zr * yt) / J
        self.sy = (xr * zt - zr * xt) / J
        self.sz = -(xr * yt - yr * xt) / J
        self.tx = (yr * zs - zr * ys) / J
        self.ty = -(xr * zs - zr * xs) / J
        self.tz = (xr * ys - yr * xs) / J
        # outward normals (mesh_3d_core.cpp:237-306 / book Normals3D)
        nx = np.stack([-self.tx, -self.sx, self.rx + self.sx + self.tx, -self.rx], axis=1)
        ny = np.stack([-self.ty, -self.sy, self.ry + self.sy + self.ty, -self.ry], axis=1)
        nz = np.stack([-self.tz, -self.sz, self.rz + self.sz + self.tz, -self.rz], axis=1)
        mag = np.sqrt(nx * nx + ny * ny + nz * nz)
        self.NX, self.NY, self.NZ = nx / mag, ny / mag, nz / mag
        self.sJ = mag * J[:, None]
        self.Fscale = self.sJ / J[:, None]
        self.dt_scale = 1 / (np.max(self.Fscale) * N * N)
        self.vmapM, self.vmapP, self.vmapF = self._vmaps()
        if high_order:
            self.high_PX, self.high_PY, self.high_PZ = self._points(v, ref.high_rst)

    @staticmethod
    def _points(v, rst):
        # x = sum_q lambda_q(r, s, t) v_q with the affine weights
        # lambda = (-(r+s+t+1), r+1, s+1, t+1) / 2: one (K,4) x (4,Np) product
        # per coordinate
        r, s, t = rst[:, 0], rst[:, 1], rst[:, 2]
        lam = 0.5 * np.stack([-(r + s + t + 1), r + 1, s + 1, t + 1])        # (4,Np)
        return [np.stack([v[q][:, d] for q in range(4)], axis=1) @ lam for d in range(3)]

    def _vmaps(self):
        ref, K, Np, Nfp = self.ref, self.Nelem, self.Np, self.Nfp
        e = np.arange(K, dtype=np.int64)
        vmapM = e[:, None, None] * Np + ref.Fmask[None, :, :].astype(np.int64)   # (K,4,Nfp)
        EtoE = self.EtoE.astype(np.int64)
        EtoF = self.EtoF.astype(np.int64)
        vmapP = vmapM.copy()
        vmapF = e[:, None] * 4 + np.arange(4)[None, :]
        inner = EtoE >= 0
        if np.any(inner):
            T, perms = _face_node_perm(ref)
            cls = self.box.vertex_class[self.box.EtoV.astype(np.int64)]          # (K,4)
            ee, ff = np.nonzero(inner)
            e2, f2 = EtoE[ee, ff], EtoF[ee, ff]
            mine = cls[ee][np.arange(len(ee))[:, None], FACE_VERTS[ff]]        # (n,3)
            theirs = cls[e2][np.arange(len(ee))[:, None], FACE_VERTS[f2]]      # (n,3)
            # p such that theirs[perm[k]] == mine[k]
            pidx = np.full(len(ee), -1, np.int64)
            for p, pi in enumerate(perms):
                ok = np.all(theirs[:, list(pi)] == mine, axis=1)
                pidx[ok] = p
            if np.any(pidx < 0):
                raise AssertionError("neighbour faces do not share their vertices")
            jpos = T[ff, f2, pidx]                                             # (n,Nfp)
            vmapP[ee, ff] = e2[:, None] * Np + ref.Fmask[f2[:, None], jpos]
            vmapF[ee, ff] = e2 * 4 + f2
        return vmapM.astype(np.int32), vmapP.astype(np.int32), vmapF.astype(np.int32)

    def calc_spatial_h(self, verbose=0):
        """min and max over elements of the inscribed-sphere diameter
        6 V / (total face area) (mesh_3d_core.cpp:444-465)."""
        V = self.box.VXYZ[self.box.EtoV.astype(np.int64)]            # (K,4,3)
        vol = np.abs(np.einsum("ki,ki->k", V[:, 1] - V[:, 0],
                               np.cross(V[:, 2] - V[:, 0], V[:, 3] - V[:, 0]))) / 6
        area = np.zeros(len(V))
        for f in FACE_VERTS:
            a, b, c = V[:, f[0]], V[:, f[1]], V[:, f[2]]
            area += 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)
        h = 6 * vol / area
        if verbose >= 1:
            print(f"min(h) ={h.min():1.5f}, max(h) ={h.max():1.5f}")
        return h.min(), h.max()

    # -- arrays in the datain layout --------------------------------------
    def datain_arrays(self):
        """Dict of every mesh array the solver reads, named as the
        reference's ``datain/*.bin`` files (dglm_3d_launcher.py:85-124)."""
        return {
            "dim": np.array([self.Nelem], np.int32),
            "EtoB": self.EtoB, "vmapP": self.vmapP, "vmapF": self.vmapF,
            "Fmask": self.ref.Fmask,
            "WDr": self.ref.WDr, "WDs": self.ref.WDs, "WDt": self.ref.WDt,
            "LIFT": self.ref.LIFT,
            "Fscale": self.Fscale, "rx": self.rx, "ry": self.ry, "rz": self.rz,
            "sx": self.sx, "sy": self.sy, "sz": self.sz,
            "tx": self.tx, "ty": self.ty, "tz": self.tz,
            "nx": self.NX, "ny": self.NY, "nz": self.NZ,
            "px": self.PX, "py": self.PY, "pz": self.PZ,
        }


def compact_face_maps(vmapP, ref, Np):
    """Compact form of a face map: per face (e, f) the neighbour element
    EtoE, its face EtoF and an orientation index EtoR into the table T of
    _face_node_perm, with vmapP[e, f, j] = EtoE Np + Fmask[EtoF, T[f, EtoF,
    EtoR, j]].  Derived from vmapP alone (any datain/vmapP.bin of this
    order); faces mapped onto themselves (vmapP = vmapM) get (e, f, 0).
    6 bytes per face instead of 4 Nfp.  Raises ValueError when a face's
    trace is not one whole face of one element."""
    Nfp = ref.Nfp
    vP = np.asarray(vmapP, dtype=np.int64).reshape(-1, 4, Nfp)
    e2 = vP // Np
    if np.any(e2 != e2[:, :, :1]):
        raise ValueError("a face's trace spans several elements")
    local = vP % Np
    T, _ = _face_node_perm(ref)
    EtoF = np.full(vP.shape[:2], -1, np.int64)
    jpos = np.zeros_like(local)
    for g in range(4):
        inv = np.full(Np, -1, np.int64)
        inv[ref.Fmask[g]] = np.arange(Nfp)
        pos = inv[local]
        whole = np.all(pos >= 0, axis=2)
        EtoF[whole] = g
        jpos[whole] = pos[whole]
    if np.any(EtoF < 0):
        raise ValueError("a face's trace is not one face of its neighbour")
    f = np.broadcast_to(np.arange(4), EtoF.shape)
    cand = T[f, EtoF]                                               # (K,4,6,Nfp)
    match = np.all(cand == jpos[:, :, None, :], axis=3)             # (K,4,6)
    if not np.all(match.any(axis=2)):
        raise ValueError("a face's node order is no rotation or reflection of its neighbour's")
    EtoR = match.argmax(axis=2)
    return e2[:, :, 0].astype(np.int32), EtoF.astype(np.uint8), EtoR.astype(np.uint8)


def expand_face_maps(EtoE, EtoF, EtoR, ref, Np):
    """vmapP (K, 4, Nfp) int32 from the compact form of compact_face_maps."""
    T, _ = _face_node_perm(ref)
    EtoE, EtoF, EtoR = (np.asarray(x, dtype=np.int64) for x in (EtoE, EtoF, EtoR))
    f = np.broadcast_to(np.arange(4), EtoF.shape)
    j2 = T[f, EtoF, EtoR]                                           # (K,4,Nfp)
    return (EtoE[:, :, None] * Np + ref.Fmask[EtoF[:, :, None], j2]).astype(np.int32)


def uniform_mesh(N, n, interpN=2, high_order=False, lo=0.0, hi=1.0, bc=None):
    """Periodic (by default) unit-cube mesh of n^3 hexahedra x 6 tets."""
    box = UniformBox(n + 1, n + 1, n + 1, lo, hi, lo, hi, lo, hi, bc=bc)
    return Mesh3D(N, box, interpN=interpN, high_order=high_order)
