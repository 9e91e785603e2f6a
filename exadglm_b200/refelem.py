"""Reference tetrahedron: nodes, orthonormal basis and the DG operators.

The solver consumes four dense operators per polynomial order N
(``WDr, WDs, WDt`` of shape (Np, Np) and ``LIFT`` of shape (Np, 4*Nfp)) plus
the face-node table ``Fmask`` (4, Nfp).  The reference builds them once per N
in mpmath at 21 significant digits and stores the float64 rounding
(dim3/src/python/tetra.py:96-301, operator_3d_ref.py:20-262,
operator_3d_face.py:74-271).  This module rebuilds them from the published
construction -- Warburton's warp-and-blend nodes (T. Warburton, "An explicit
construction of interpolation nodes on the simplex", J. Eng. Math. 2006) and
the orthonormal Dubiner/Koornwinder basis with the nodal operators of
Hesthaven & Warburton, "Nodal Discontinuous Galerkin Methods" (2008), ch. 6
and 10 -- evaluated in x87 extended precision (64-bit mantissa), so that the
float64 results agree with the reference's stored matrices to a few ulp.

Node numbering, face-node order and the rounding of stored matrices follow
the reference, because they are part of the data format the solver reads:

* equidistant seed nodes: r fastest, then s, then t, seeded from float64
  values of ``-1 + 2*(q-1)/N`` (tetra.py:96-111);
* the optimised blending parameters per N (tetra.py:122-124, the published
  table of the book, Table 6.1);
* Fmask rows come in increasing node order, with the row order reversed on
  faces 0 and 3 (operator_3d_face.py:74-123);
* entries smaller than ``max(matrix)*eps`` are flushed to zero before storage
  (utils/src/python/io_mp_mats.py:18-22).
"""
from __future__ import annotations

import functools
import math

import numpy as np

LD = np.longdouble
TOL = 1e-15
NODETOL = 1e-12

# Optimised warp-and-blend parameter for N = 1..15 (book Table 6.1; same
# values the reference seeds from, tetra.py:122-124).
_ALPHA_OPT = (0.0, 0.0, 0.0, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577, 1.1603,
              1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655)

_PI = LD("3.14159265358979323846264338327950288")


def dims(N: int):
    """Return (Np, Nfp) for polynomial order N."""
    return (N + 1) * (N + 2) * (N + 3) // 6, (N + 1) * (N + 2) // 2


# ---------------------------------------------------------------------------
# small extended-precision linear algebra
# ---------------------------------------------------------------------------

def ld_inv(A):
    """Inverse of a square matrix by Gauss-Jordan with partial pivoting,
    carried out in long double (numpy.linalg has no long-double kernels)."""
    A = np.array(A, dtype=LD)
    n = A.shape[0]
    M = np.concatenate([A, np.eye(n, dtype=LD)], axis=1)
    for c in range(n):
        p = c + int(np.argmax(np.abs(M[c:, c])))
        if M[p, c] == 0:
            raise np.linalg.LinAlgError("singular matrix")
        if p != c:
            M[[c, p]] = M[[p, c]]
        M[c] /= M[c, c]
        col = M[:, c].copy()
        col[c] = 0
        M -= np.outer(col, M[c])
    return M[:, n:]


def ld_matmul(A, B):
    """Matrix product in long double (numpy's matmul keeps the dtype)."""
    return np.matmul(np.asarray(A, dtype=LD), np.asarray(B, dtype=LD))


# ---------------------------------------------------------------------------
# orthonormal Jacobi polynomials and Gauss-Lobatto nodes
# ---------------------------------------------------------------------------

def jacobi_p(x, alpha: int, beta: int, n: int):
    """Orthonormal Jacobi polynomial P_n^(alpha,beta) at x (long double),
    by the three-term recurrence (book eq. A.1-A.4)."""
    x = np.asarray(x, dtype=LD)
    a, b = alpha, beta
    g0 = LD(2) ** (a + b + 1) / LD(a + b + 1) * LD(math.factorial(a)) * \
        LD(math.factorial(b)) / LD(math.factorial(a + b))
    p_prev = np.full(x.shape, 1 / np.sqrt(g0), dtype=LD)
    if n == 0:
        return p_prev
    g1 = LD((a + 1) * (b + 1)) / LD(a + b + 3) * g0
    p_cur = (LD(a + b + 2) * x / 2 + LD(a - b) / 2) / np.sqrt(g1)
    if n == 1:
        return p_cur
    a_old = LD(2) / LD(a + b + 2) * np.sqrt(LD((a + 1) * (b + 1)) / LD(a + b + 3))
    for i in range(1, n):
        h1 = LD(2 * i + a + b)
        a_new = LD(2) / (h1 + 2) * np.sqrt(
            LD((i + 1) * (i + 1 + a + b) * (i + 1 + a) * (i + 1 + b)) / (h1 + 1) / (h1 + 3))
        b_new = -LD(a * a - b * b) / h1 / (h1 + 2)
        p_next = (-a_old * p_prev + (x - b_new) * p_cur) / a_new
        p_prev, p_cur = p_cur, p_next
        a_old = a_new
    return p_cur


def grad_jacobi_p(x, alpha: int, beta: int, n: int):
    """d/dx of the orthonormal Jacobi polynomial (book eq. A.2)."""
    x = np.asarray(x, dtype=LD)
    if n == 0:
        return np.zeros(x.shape, dtype=LD)
    return np.sqrt(LD(n * (n + alpha + beta + 1))) * jacobi_p(x, alpha + 1, beta + 1, n - 1)


def gauss_jacobi_nodes(n: int, alpha: int, beta: int):
    """Roots of P_{n+1}^(alpha,beta): Golub-Welsch in float64, then Newton
    polishing in long double."""
    if n == 0:
        return np.array([LD(alpha - beta) / LD(alpha + beta + 2)], dtype=LD)
    k = np.arange(n + 1, dtype=np.float64)
    h1 = 2 * k + alpha + beta
    with np.errstate(divide="ignore", invalid="ignore"):
        diag = -0.5 * (alpha ** 2 - beta ** 2) / (h1 + 2) / h1
    if alpha + beta == 0:
        diag[0] = 0.0
    kp = k[:-1] + 1
    off = 2 / (h1[:-1] + 2) * np.sqrt(kp * (kp + alpha + beta) * (kp + alpha) * (kp + beta)
                                      / (h1[:-1] + 1) / (h1[:-1] + 3))
    J = np.diag(diag) + np.diag(off, 1) + np.diag(off, -1)
    x = np.sort(np.linalg.eigvalsh(J)).astype(LD)
    for _ in range(6):
        f = jacobi_p(x, alpha, beta, n + 1)
        df = grad_jacobi_p(x, alpha, beta, n + 1)
        x = x - f / df
    if (n + 1) % 2 == 1:
        x[n // 2] = 0
    return x


def gll_nodes(N: int):
    """Gauss-Lobatto-Legendre nodes on [-1, 1], ascending."""
    x = np.empty(N + 1, dtype=LD)
    x[0], x[N] = -1, 1
    if N > 1:
        x[1:N] = gauss_jacobi_nodes(N - 2, 1, 1)
    return x


# ---------------------------------------------------------------------------
# warp & blend nodes (Warburton 2006)
# ---------------------------------------------------------------------------

def _warp_factor(N: int, r):
    """Edge warp divided by the edge bubble (1 - r^2), evaluated in the
    factored form that stays finite at r = +-1:
        w(r) = sum_i (x_i^GLL - x_i^eq) * l_i(r) / (1 - r^2)
    where l_i is the Lagrange basis on the N+1 equidistant points."""
    r = np.asarray(r, dtype=LD)
    xg = -gll_nodes(N)          # descending, to pair with the equidistant list
    xe = np.array([LD(-1) + LD(2 * (N + 1 - i)) / LD(N) for i in range(1, N + 2)], dtype=LD)
    w = np.zeros(r.shape, dtype=LD)
    for i in range(N + 1):
        d = np.full(r.shape, xg[i] - xe[i], dtype=LD)
        for j in range(1, N):          # interior equidistant points only
            if j != i:
                d = d * (r - xe[j]) / (xe[i] - xe[j])
        if i != 0:
            d = -d / (xe[i] - xe[0])
        if i != N:
            d = d / (xe[i] - xe[N])
        w = w + d
    return w


def _face_shift(N: int, alpha, L1, L2, L3):
    """Tangential warp of the 2-D face with barycentric coordinates L1..L3."""
    b1, b2, b3 = L2 * L3, L1 * L3, L1 * L2
    w1 = b1 * 4 * _warp_factor(N, L3 - L2) * (1 + (alpha * L1) ** 2)
    w2 = b2 * 4 * _warp_factor(N, L1 - L3) * (1 + (alpha * L2) ** 2)
    w3 = b3 * 4 * _warp_factor(N, L2 - L1) * (1 + (alpha * L3) ** 2)
    c, s = LD(-0.5), np.sqrt(LD(3)) / 2     # cos/sin of 2*pi/3; 4*pi/3 -> (c, -s)
    return w1 + c * w2 + c * w3, s * w2 - s * w3


def _equidistant_rst(N: int):
    """Equidistant seed nodes, r fastest; each coordinate is the float64
    value of -1 + 2*(q-1)/N, as the reference seeds its construction."""
    pts = []
    for n in range(1, N + 2):
        for m in range(1, N + 3 - n):
            for q in range(1, N + 4 - n - m):
                pts.append((-1 + (q - 1) * 2 / N, -1 + (m - 1) * 2 / N, -1 + (n - 1) * 2 / N))
    return np.array(pts, dtype=np.float64).astype(LD)


def _tet_vertices():
    s3, s6 = np.sqrt(LD(3)), np.sqrt(LD(6))
    return (np.array([-1, -1 / s3, -1 / s6], dtype=LD), np.array([1, -1 / s3, -1 / s6], dtype=LD),
            np.array([0, 2 / s3, -1 / s6], dtype=LD), np.array([0, 0, 3 / s6], dtype=LD))


def nodes_equilateral(N: int):
    """Warp & blend nodes in the equilateral tetrahedron, shape (Np, 3)."""
    alpha = LD(_ALPHA_OPT[N - 1]) if N <= 15 else LD(1)
    rst = _equidistant_rst(N)
    r, s, t = rst[:, 0], rst[:, 1], rst[:, 2]
    L1, L2 = (1 + t) / 2, (1 + s) / 2
    L3, L4 = -(1 + r + s + t) / 2, (1 + r) / 2
    v1, v2, v3, v4 = _tet_vertices()
    t1 = np.array([v2 - v1, v2 - v1, v3 - v2, v3 - v1], dtype=LD)
    t2 = np.array([v3 - (v1 + v2) / 2, v4 - (v1 + v2) / 2,
                   v4 - (v2 + v3) / 2, v4 - (v1 + v3) / 2], dtype=LD)
    t1 /= np.sqrt((t1 ** 2).sum(axis=1))[:, None]
    t2 /= np.sqrt((t2 ** 2).sum(axis=1))[:, None]
    xyz = np.outer(L3, v1) + np.outer(L4, v2) + np.outer(L2, v3) + np.outer(L1, v4)
    shift = np.zeros_like(xyz)
    faces = ((L1, L2, L3, L4), (L2, L1, L3, L4), (L3, L1, L4, L2), (L4, L1, L3, L2))
    for f, (La, Lb, Lc, Ld) in enumerate(faces):
        w1, w2 = _face_shift(N, alpha, Lb, Lc, Ld)
        blend = Lb * Lc * Ld
        denom = (Lb + La / 2) * (Lc + La / 2) * (Ld + La / 2)
        ok = denom > TOL
        blend = np.where(ok, (1 + (alpha * La) ** 2) * blend / np.where(ok, denom, 1), blend)
        dshift = np.outer(w1, t1[f]) + np.outer(w2, t2[f])
        on_face = (La < TOL) & (((Lb > TOL).astype(int) + (Lc > TOL) + (Ld > TOL)) < 3)
        shift = np.where(on_face[:, None], dshift, shift + blend[:, None] * dshift)
    return xyz + shift


def equilateral_to_rst(xyz):
    """Map equilateral-tetrahedron points to the reference (r, s, t)
    tetrahedron with vertices (-1,-1,-1), (1,-1,-1), (-1,1,-1), (-1,-1,1)."""
    v1, v2, v3, v4 = _tet_vertices()
    A = np.stack([(v2 - v1) / 2, (v3 - v1) / 2, (v4 - v1) / 2], axis=1)
    rhs = np.asarray(xyz, dtype=LD) - (v2 + v3 + v4 - v1) / 2
    return ld_matmul(rhs, ld_inv(A).T)


def rst_to_abc(rst):
    """Collapsed coordinates (a, b, c) used by the orthonormal basis."""
    r, s, t = rst[:, 0], rst[:, 1], rst[:, 2]
    st = s + t
    a = np.where(np.abs(st) > TOL, -2 * (1 + r) / np.where(np.abs(st) > TOL, st, 1) - 1, -1)
    b = np.where(np.abs(t - 1) > TOL, 2 * (1 + s) / np.where(np.abs(t - 1) > TOL, 1 - t, 1) - 1, -1)
    return np.stack([a.astype(LD), b.astype(LD), t], axis=1)


# ---------------------------------------------------------------------------
# orthonormal simplex basis and its gradient
# ---------------------------------------------------------------------------

def _modes3d(N: int):
    return [(i, j, k) for i in range(N + 1) for j in range(N - i + 1) for k in range(N - i - j + 1)]


def basis3d(abc, i, j, k):
    a, b, c = abc[:, 0], abc[:, 1], abc[:, 2]
    return (2 * np.sqrt(LD(2)) * jacobi_p(a, 0, 0, i) * jacobi_p(b, 2 * i + 1, 0, j)
            * (1 - b) ** i * jacobi_p(c, 2 * (i + j) + 2, 0, k) * (1 - c) ** (i + j))


def grad_basis3d(abc, i, j, k):
    """(d/dr, d/ds, d/dt) of the orthonormal mode (i, j, k) (book GradSimplex3DP)."""
    a, b, c = abc[:, 0], abc[:, 1], abc[:, 2]
    fa, dfa = jacobi_p(a, 0, 0, i), grad_jacobi_p(a, 0, 0, i)
    gb, dgb = jacobi_p(b, 2 * i + 1, 0, j), grad_jacobi_p(b, 2 * i + 1, 0, j)
    hc, dhc = jacobi_p(c, 2 * (i + j) + 2, 0, k), grad_jacobi_p(c, 2 * (i + j) + 2, 0, k)
    hb, hcm = (1 - b) / 2, (1 - c) / 2
    dr = dfa * gb * hc
    if i > 0:
        dr = dr * hb ** (i - 1)
    if i + j > 0:
        dr = dr * hcm ** (i + j - 1)
    ds = (1 + a) / 2 * dr
    tmp = dgb * hb ** i
    if i > 0:
        tmp = tmp + (-LD(i) / 2) * (gb * hb ** (i - 1))
    if i + j > 0:
        tmp = tmp * hcm ** (i + j - 1)
    tmp = fa * tmp * hc
    ds = ds + tmp
    dt = (1 + a) / 2 * dr + (1 + b) / 2 * tmp
    tmp = dhc * hcm ** (i + j)
    if i + j > 0:
        tmp = tmp - LD(i + j) / 2 * hc * hcm ** (i + j - 1)
    tmp = fa * gb * tmp * hb ** i
    dt = dt + tmp
    scale = LD(2) ** (2 * i + j) * LD(2) * np.sqrt(LD(2))   # 2^(2i+j+1.5)
    return dr * scale, ds * scale, dt * scale


def basis2d(a, b, i, j):
    return np.sqrt(LD(2)) * jacobi_p(a, 0, 0, i) * jacobi_p(b, 2 * i + 1, 0, j) * (1 - b) ** i


def vandermonde3d(N, abc):
    return np.stack([basis3d(abc, *m) for m in _modes3d(N)], axis=1)


def vandermonde2d(N, a, b):
    return np.stack([basis2d(a, b, i, j) for i in range(N + 1) for j in range(N - i + 1)], axis=1)


# ---------------------------------------------------------------------------
# face masks
# ---------------------------------------------------------------------------

def _rows(idx, N):
    """Split a face's node list into its N+1 lattice rows (lengths N+1..1)."""
    out, k = [], 0
    for n in range(N + 1, 0, -1):
        out.append(list(idx[k:k + n]))
        k += n
    return out


def _turn(rows):
    """Rotate a triangular row layout by one vertex: new[k][m] = old[n-1-k-m][k]."""
    n = len(rows)
    return [[rows[n - 1 - k - m][k] for m in range(n - k)] for k in range(n)]


def _flip(rows):
    return [r[::-1] for r in rows]


def face_masks(N: int, rst64):
    """Fmask (4, Nfp) and the three rotated, inverted orders FmaskP (4, 3, Nfp).
    Faces: 0 t=-1, 1 s=-1, 2 r+s+t=-1, 3 r=-1."""
    r, s, t = rst64[:, 0], rst64[:, 1], rst64[:, 2]
    faces = [np.where(np.abs(t + 1) < NODETOL)[0], np.where(np.abs(s + 1) < NODETOL)[0],
             np.where(np.abs(r + s + t + 1) < NODETOL)[0], np.where(np.abs(r + 1) < NODETOL)[0]]
    Np, Nfp = dims(N)
    Fmask = np.zeros((4, Nfp), np.int32)
    FmaskP = np.zeros((4, 3, Nfp), np.int32)
    for f, idx in enumerate(faces):
        assert len(idx) == Nfp, "face node detection failed"
        rows = _rows(idx, N)
        if f in (0, 3):
            rows = _flip(rows)
        r1 = _turn(rows)
        r2 = _turn(r1)
        Fmask[f] = sum(rows, [])
        for rot, rr in enumerate((rows, r1, r2)):
            FmaskP[f, rot] = sum(_flip(rr), [])
    return Fmask, FmaskP


def flush_tiny(arr):
    """Zero the entries below max(arr)*eps, as the reference does before
    writing its float64 matrices."""
    arr = np.array(arr, dtype=np.float64)
    tol = arr.max() * np.finfo(np.float64).eps
    arr[np.abs(arr) < tol] = 0
    return arr


# ---------------------------------------------------------------------------
# operator bundle
# ---------------------------------------------------------------------------

class RefElement:
    """All reference-element data for order N (float64 views of long-double
    computations).

    Attributes follow the reference's names: ``rst`` (Np,3), ``Fmask``
    (4,Nfp), ``FmaskP`` (4,3,Nfp), ``M``, ``Dr/Ds/Dt``, ``WDr/WDs/WDt``
    (Np,Np), ``Emat``/``LIFT`` (Np,4*Nfp), ``interpM`` (high_Np,Np),
    ``high_M`` and ``high_rst`` for the L2 error at order N+interpN.
    """

    def __init__(self, N: int, interpN: int = 2):
        if N < 1:
            raise ValueError("N must be >= 1")
        self.N = N
        self.Np, self.Nfp = dims(N)
        self.Nface, self.Nrot = 4, 3
        self.interpN = interpN
        self.high_N = N + interpN
        self.high_Np = dims(self.high_N)[0]
        b = _build(N)
        self.rst_ld, self.abc = b["rst"], b["abc"]
        self.rst = flush_tiny(self.rst_ld)
        self.xyz = flush_tiny(b["xyz"])
        V, invV = b["V"], b["invV"]
        Vr, Vs, Vt = b["Vr"], b["Vs"], b["Vt"]
        Dr, Ds, Dt = ld_matmul(Vr, invV), ld_matmul(Vs, invV), ld_matmul(Vt, invV)
        M = ld_matmul(invV.T, invV)
        invM = ld_matmul(V, V.T)
        self.M = flush_tiny(M)
        self.Dr, self.Ds, self.Dt = flush_tiny(Dr), flush_tiny(Ds), flush_tiny(Dt)
        self.WDr = flush_tiny(ld_matmul(ld_matmul(invM, Dr.T), M))
        self.WDs = flush_tiny(ld_matmul(ld_matmul(invM, Ds.T), M))
        self.WDt = flush_tiny(ld_matmul(ld_matmul(invM, Dt.T), M))
        self.Fmask, self.FmaskP = face_masks(N, self.rst)
        Emat = np.zeros((self.Np, 4 * self.Nfp), dtype=LD)
        coords = ((0, 1), (0, 2), (1, 2), (1, 2))     # collapsed coords spanning each face
        for f in range(4):
            idx = self.Fmask[f]
            V2 = vandermonde2d(N, self.abc[idx, coords[f][0]], self.abc[idx, coords[f][1]])
            iV2 = ld_inv(V2)
            Emat[idx, f * self.Nfp:(f + 1) * self.Nfp] = ld_matmul(iV2.T, iV2)
        self.Emat = flush_tiny(Emat)
        self.LIFT = flush_tiny(ld_matmul(V, ld_matmul(V.T, Emat)))
        hb = _build(self.high_N)
        self.high_rst = flush_tiny(hb["rst"])
        interpV = np.stack([basis3d(hb["abc"], *m) for m in _modes3d(N)], axis=1)
        self.interpM = flush_tiny(ld_matmul(interpV, invV))
        self.high_M = flush_tiny(ld_matmul(hb["invV"].T, hb["invV"]))


@functools.lru_cache(maxsize=32)
def _build_cached(N: int):
    xyz = nodes_equilateral(N)
    rst = equilateral_to_rst(xyz)
    abc = rst_to_abc(rst)
    V = vandermonde3d(N, abc)
    invV = ld_inv(V)
    grads = [grad_basis3d(abc, *m) for m in _modes3d(N)]
    Vr = np.stack([g[0] for g in grads], axis=1)
    Vs = np.stack([g[1] for g in grads], axis=1)
    Vt = np.stack([g[2] for g in grads], axis=1)
    return dict(xyz=xyz, rst=rst, abc=abc, V=V, invV=invV, Vr=Vr, Vs=Vs, Vt=Vt)


def _build(N: int):
    return _build_cached(N)


@functools.lru_cache(maxsize=32)
def ref_element(N: int, interpN: int = 2) -> RefElement:
    """Cached RefElement for (N, interpN)."""
    return RefElement(N, interpN)
