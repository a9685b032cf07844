"""CPU oracle for the boundary-mode-analysis (port-mode) matrices — TEST INFRASTRUCTURE ONLY.

Restates, vectorised over triangles, the mixed Nedelec-2 / Lagrange-2 triangle element of
``generalized_matrix_GQ`` and its COO builder ``_matrix_builder``
(``src/emerge/_emerge/physics/microwave/assembly/generalized_eigen_hb.py:257-458``).

Element DOFs (``elements/nedleg2.py:140-150``): [e1 e2 e3 f | e1' e2' e3' f' | v1 v2 v3 | m1 m2 m3]
(first-kind edge and face functions, second-kind ones, then the vertex and edge-midpoint
Lagrange-2 functions of E_z).  With L_i = a_i + b_i x + c_i y the barycentrics of the triangle in the
port's local 2-D frame (``tri_coefficients``, :202-226), W_ij = L_i grad L_j - L_j grad L_i and
e = (i, j) a local edge in the global edge's node order:

* edge:  N_e = W_ij, N_e' = W_ij (L_i - L_j), curl N_e = 2 k_ij, curl N_e' = grad(L_i - L_j) x W_ij
  + 2 k_ij (L_i - L_j), k_ij = b_i c_j - b_j c_i  (:88-112, :175-187);
* face:  N_f = L_2 W_13 + L_1 W_23, N_f' = -(L_3 W_12 + L_2 W_13) and their curls (:114-136, :189-199);
* Lagrange: vertex L(2L - 1), edge 4 L_i L_j and their gradients (:138-172).

The 6-point rule is the reference's 8-digit Dunavant table (:232-235).  Blocks, with Ms = ur^-1
(``matinv``), Mm = er, the 2x2 upper-left parts for the transverse terms and the zz entries for
curl/E_z:  A = [[Att - k0^2 Btt, 0], [0, 0]], B = [[Dtt, Dzt^T], [Dzt, Dzz1 - k0^2 Dzz2]], both times
the triangle area.  Three properties of the reference are kept on purpose: the face rows of Att, Btt
and Dtt copy the face columns (:375-398), the face-face entries of Dtt are never filled (zero), and
the edge-length scaling ``Ls`` is reset to ones before use (:433).
"""
from __future__ import annotations

import numpy as np
from scipy.sparse import csr_matrix

from .abc2 import DPTS

NE = 14


def matinv(M: np.ndarray) -> np.ndarray:
    """(3, 3, n) complex inverse with the diagonal fast path of ``mth/optimized.py:342-370``."""
    out = np.zeros_like(M)
    off = np.abs(M[0, 1]) + np.abs(M[0, 2]) + np.abs(M[1, 0]) + np.abs(M[1, 2]) + np.abs(M[2, 0]) + np.abs(M[2, 1])
    diag = off == 0
    for i in range(3):
        out[i, i, diag] = 1.0 / M[i, i, diag]
    g = ~diag
    if g.any():
        out[:, :, g] = np.linalg.inv(M[:, :, g].transpose(2, 0, 1)).transpose(1, 2, 0)
    return out


def tri_coefficients(x: np.ndarray, y: np.ndarray):
    """x, y (nt, 3) vertex coordinates -> a, b, c (nt, 3) sign-corrected, area (nt,)."""
    x1, x2, x3 = x.T
    y1, y2, y3 = y.T
    a = np.stack([x2 * y3 - y2 * x3, x3 * y1 - y3 * x1, x1 * y2 - y1 * x2], 1)
    b = np.stack([y2 - y3, y3 - y1, y1 - y2], 1)
    c = np.stack([x3 - x2, x1 - x3, x2 - x1], 1)
    sA = 0.5 * ((x1 - x3) * (y2 - y1) - (x1 - x2) * (y3 - y1))
    s = np.sign(sA)[:, None]
    return a * s, b * s, c * s, np.abs(sA)


def local_edge_map(tris: np.ndarray, edges: np.ndarray, tri_to_edge: np.ndarray) -> np.ndarray:
    """(2, 3, nt): local vertex slots of each triangle edge's two global nodes (``local_tri_to_edgeid``)."""
    out = np.zeros((2, 3, tris.shape[1]), dtype=np.int64)
    for k in range(3):
        ge = edges[:, tri_to_edge[k]]
        for s in range(2):
            out[s, k] = np.argmax(tris == ge[s][None, :], axis=0)
    return out


def _dot(u, M, v):
    """sum_w W_w * (u . (M v)) per triangle: u, v (2, nt, np), M (2, 2, nt) complex."""
    Mv0 = M[0, 0][:, None] * v[0] + M[0, 1][:, None] * v[1]
    Mv1 = M[1, 0][:, None] * v[0] + M[1, 1][:, None] * v[1]
    return np.sum(DPTS[0][None, :] * (u[0] * Mv0 + u[1] * Mv1), axis=1)


def _sdot(u, m, v):
    """sum_w u * (m v) * W for scalars u, v (nt, np), m (nt,)."""
    return np.sum(u * (m[:, None] * v) * DPTS[0][None, :], axis=1)


def element_matrices(local_nodes, tris, edges, tri_to_edge, er, ur, k0):
    """A, B (nt, 14, 14) complex for every triangle."""
    nt = tris.shape[1]
    x = local_nodes[0][tris].T
    y = local_nodes[1][tris].T
    a, b, c, area = tri_coefficients(x, y)
    a, b, c = a / (2 * area[:, None]), b / (2 * area[:, None]), c / (2 * area[:, None])
    xs = x[:, 0:1] * DPTS[1] + x[:, 1:2] * DPTS[2] + x[:, 2:3] * DPTS[3]
    ys = y[:, 0:1] * DPTS[1] + y[:, 1:2] * DPTS[2] + y[:, 2:3] * DPTS[3]
    L = [a[:, i:i + 1] + b[:, i:i + 1] * xs + c[:, i:i + 1] * ys for i in range(3)]
    g = [(b[:, i:i + 1], c[:, i:i + 1]) for i in range(3)]
    ar = np.arange(nt)

    def W(i, j):
        Li, Lj = L[i], L[j]
        gi, gj = g[i], g[j]
        return np.stack([Li * gj[0] - Lj * gi[0], Li * gj[1] - Lj * gi[1]])

    def k(i, j):
        return g[i][0] * g[j][1] - g[j][0] * g[i][1]

    def cross(gr, V):
        return gr[0] * V[1] - gr[1] * V[0]

    emap = local_edge_map(tris, edges, tri_to_edge)
    Lst = np.stack(L)                       # (3, nt, np)
    bst = np.stack([b, c])                  # (2, nt, 3)
    N = np.zeros((8, 2, nt, len(DPTS[0])))
    curl = np.zeros((8, nt, len(DPTS[0])))
    lag = np.zeros((6, nt, len(DPTS[0])))
    glag = np.zeros((6, 2, nt, len(DPTS[0])))
    for e in range(3):
        i1, i2 = emap[0, e], emap[1, e]
        L1, L2 = Lst[i1, ar], Lst[i2, ar]
        g1 = (bst[0, ar, i1][:, None], bst[1, ar, i1][:, None])
        g2 = (bst[0, ar, i2][:, None], bst[1, ar, i2][:, None])
        Wv = np.stack([L1 * g2[0] - L2 * g1[0], L1 * g2[1] - L2 * g1[1]])
        kk = g1[0] * g2[1] - g2[0] * g1[1]
        N[e] = Wv
        N[4 + e] = Wv * (L1 - L2)
        curl[e] = 2 * kk * np.ones_like(L1)
        curl[4 + e] = (g1[0] - g2[0]) * Wv[1] - (g1[1] - g2[1]) * Wv[0] + 2 * kk * (L1 - L2)
        lag[3 + e] = 4 * L1 * L2
        glag[3 + e] = 4 * np.stack([g1[0] * L2 + g2[0] * L1, g1[1] * L2 + g2[1] * L1])
        Lv = L[e]
        lag[e] = Lv * (2 * Lv - 1)
        glag[e] = np.stack([g[e][0] * (4 * Lv - 1), g[e][1] * (4 * Lv - 1)])
    W13, W23, W12 = W(0, 2), W(1, 2), W(0, 1)
    N[3] = L[1] * W13 + L[0] * W23
    N[7] = -(L[2] * W12 + L[1] * W13)
    curl[3] = cross(g[1], W13) + 2 * L[1] * k(0, 2) + cross(g[0], W23) + 2 * L[0] * k(1, 2)
    curl[7] = -(cross(g[2], W12) + 2 * L[2] * k(0, 1) + cross(g[1], W13) + 2 * L[1] * k(0, 2))

    Ms = matinv(np.asarray(ur, dtype=np.complex128))
    Mm = np.asarray(er, dtype=np.complex128)
    Ms2, Mm2, Msz, Mmz = Ms[:2, :2], Mm[:2, :2], Ms[2, 2], Mm[2, 2]
    Att = np.zeros((nt, 8, 8), complex)
    Btt = np.zeros_like(Att)
    Dtt = np.zeros_like(Att)
    Dzt = np.zeros((nt, 6, 8), complex)
    Dzz = np.zeros((nt, 6, 6), complex)
    face = (3, 7)
    for i in range(8):
        for j in range(8):
            if i in face and j not in face:      # face rows copy the face columns
                ii, jj = j, i
            else:
                ii, jj = i, j
            Att[:, i, j] = _sdot(curl[ii], Msz, curl[jj])
            Btt[:, i, j] = _dot(N[ii], Mm2, N[jj])
            if not (i in face and j in face):
                Dtt[:, i, j] = _dot(N[ii], Ms2, N[jj])
    for r in range(6):
        for j in range(8):
            Dzt[:, r, j] = _dot(glag[r], Ms2, N[j])
        for s in range(6):
            Dzz[:, r, s] = _dot(glag[r], Ms2, glag[s]) - k0 ** 2 * _sdot(lag[r], Mmz, lag[s])
    A = np.zeros((nt, NE, NE), complex)
    B = np.zeros((nt, NE, NE), complex)
    A[:, :8, :8] = Att - k0 ** 2 * Btt
    B[:, :8, :8] = Dtt
    B[:, 8:, :8] = Dzt
    B[:, :8, 8:] = Dzt.transpose(0, 2, 1)
    B[:, 8:, 8:] = Dzz
    return A * area[:, None, None], B * area[:, None, None]


def matrix_builder(local_nodes, tris, edges, tri_to_field, ur, er, k0):
    """The reference's ``_matrix_builder`` outputs: dataE, dataB (196 nt,), rows, cols."""
    A, B = element_matrices(local_nodes, tris, edges, tri_to_field[:3], er, ur, k0)
    idx = tri_to_field.T                                     # (nt, 14)
    rows = np.repeat(idx, NE, axis=1).ravel()
    cols = np.tile(idx, (1, NE)).ravel()
    return A.reshape(-1), B.reshape(-1), rows, cols


def generalized_eigenvalue_matrix(local_nodes, tris, edges, tri_to_field, n_field, er, ur, k0):
    dE, dB, r, c = matrix_builder(local_nodes, tris, edges, tri_to_field, ur, er, k0)
    return (csr_matrix((dE, (r, c)), shape=(n_field, n_field)),
            csr_matrix((dB, (r, c)), shape=(n_field, n_field)))
