"""CPU oracle for the auxiliary nodal space and the preconditioner network — TEST INFRASTRUCTURE ONLY.

* :func:`gradient_matrix` fits, per tet, the gradients of the second-order nodal functions (vertex
  hats L_v and edge functions L_a L_b) in the reference's Nedelec-2 basis by least squares at
  sample points.  The basis is evaluated exactly as ``ned2_tet_interp`` does
  (``src/emerge/_emerge/elements/ned2_interp.py:142-300``: edge functions
  ``l (E1 L1 + E2 L2)(L2 grad L1 - L1 grad L2)``, face functions
  ``-E1 l_13 L2 (L3 grad L1 - L1 grad L3) + E2 l_12 L3 (L2 grad L1 - L1 grad L2)`` with the local
  vertex order of the sorted global edge / triangle), so this is an independent check of the
  closed-form discrete gradient the library builds per entity.
* :func:`aux_diagonals` is diag(Gᵀ X G) with SciPy.
* :func:`mpnn_forward` / :func:`mpnn_backward` restate the network of ``emfem_mpnn_*`` in float64
  numpy, for the gradient check of the GPU training kernels.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

C = 32
L = 4
NPARAMS = 2 * C + L * 4 * C * C + 2 * C


def _local(tets: np.ndarray, ids_glob: np.ndarray) -> np.ndarray:
    """Local vertex slot (0..3) of each global node id in ids_glob (k, nt)."""
    out = np.zeros_like(ids_glob)
    for k in range(ids_glob.shape[0]):
        out[k] = np.argmax(tets == ids_glob[k][None, :], axis=0)
    return out


def basis_values(mesh, field, bary: np.ndarray):
    """(nt, npts, 20, 3) basis vectors at barycentric points bary (npts, 4), and the barycentric
    gradients (nt, 4, 3)."""
    nodes, tets = mesh.nodes, mesh.tets
    nt = tets.shape[1]
    X = nodes[:, tets]                                   # (3, 4, nt)
    Mm = np.ones((nt, 4, 4))
    Mm[:, :, 1:] = X.transpose(2, 1, 0)
    grad = np.linalg.inv(Mm)[:, 1:, :].transpose(0, 2, 1)      # (nt, 4, 3)
    npts = bary.shape[0]
    Lb = np.broadcast_to(bary[None], (nt, npts, 4))

    def lv(i):
        return np.take_along_axis(Lb, np.broadcast_to(i[:, None, None], (nt, npts, 1)), 2)[..., 0]

    ar = np.arange(nt)
    out = np.zeros((nt, npts, 20, 3))
    t2f, ne = field.tet_to_field, mesh.n_edges
    for ie in range(6):
        ge = mesh.edges[:, t2f[ie]]
        a, b = _local(tets, ge)
        la, lb = lv(a), lv(b)
        ga, gb = grad[ar, a], grad[ar, b]
        ln = np.linalg.norm(nodes[:, ge[0]] - nodes[:, ge[1]], axis=0)[:, None, None]
        W = lb[..., None] * ga[:, None, :] - la[..., None] * gb[:, None, :]
        out[:, :, ie] = ln * la[..., None] * W
        out[:, :, 10 + ie] = ln * lb[..., None] * W
    for jf in range(4):
        gt = mesh.tris[:, t2f[6 + jf] - ne]
        a, b, c = _local(tets, gt)
        l1, l2, l3 = lv(a), lv(b), lv(c)
        g1, g2, g3 = grad[ar, a], grad[ar, b], grad[ar, c]
        L1 = np.linalg.norm(nodes[:, gt[0]] - nodes[:, gt[2]], axis=0)[:, None, None]
        L2 = np.linalg.norm(nodes[:, gt[0]] - nodes[:, gt[1]], axis=0)[:, None, None]
        W13 = l3[..., None] * g1[:, None] - l1[..., None] * g3[:, None]
        W12 = l2[..., None] * g1[:, None] - l1[..., None] * g2[:, None]
        out[:, :, 6 + jf] = -(L1 * l2[..., None] * W13)
        out[:, :, 16 + jf] = L2 * l3[..., None] * W12
    return out, grad


def gradient_matrix(mesh, field, seed: int = 0) -> sp.csr_matrix:
    """G (N x (N_n + N_e)): column v = grad L_v, column N_n + e = grad (L_a L_b) of edge e."""
    rng = np.random.default_rng(seed)
    P = rng.dirichlet(np.ones(4), 24)
    Bv, grad = basis_values(mesh, field, P)
    nt = mesh.n_tets
    M = Bv.transpose(0, 1, 3, 2).reshape(nt, 72, 20)
    F = np.zeros((nt, 24, 3, 10))
    for a in range(4):
        F[:, :, :, a] = grad[:, a][:, None, :]
    for k, (a, b) in enumerate(((0, 1), (0, 2), (0, 3), (1, 2), (3, 1), (2, 3))):
        F[:, :, :, 4 + k] = P[None, :, a, None] * grad[:, b][:, None, :] + P[None, :, b, None] * grad[:, a][:, None, :]
    F = F.reshape(nt, 72, 10)
    Mt = M.transpose(0, 2, 1)
    Cf = np.linalg.solve(Mt @ M, Mt @ F)                  # (nt, 20, 10)
    nn, ne = mesh.n_nodes, mesh.n_edges
    rows = np.repeat(field.tet_to_field.T[:, :, None], 10, axis=2)
    aux = np.concatenate([mesh.tets.T, nn + mesh.tet_to_edge.T], axis=1)
    cols = np.repeat(aux[:, None, :], 20, axis=1)
    v = Cf.ravel()
    keep = np.abs(v) > 1e-9 * np.abs(v).max()
    r, c, v = rows.ravel()[keep], cols.ravel()[keep], v[keep]
    G = sp.coo_matrix((v, (r, c)), shape=(field.n_field, nn + ne)).tocsr()
    cnt = sp.coo_matrix((np.ones(len(v)), (r, c)), shape=G.shape).tocsr()
    G.data = G.data / cnt.data                            # entries shared by several tets agree
    return G


def aux_diagonals(G: sp.csr_matrix, X: sp.spmatrix) -> np.ndarray:
    return np.asarray((G.T @ X @ G).diagonal())


# ---------------------------------------------------------------------------- network
def unpack(params: np.ndarray):
    p = np.asarray(params, dtype=np.float64)
    o = 0
    w_in = p[o:o + 2 * C].reshape(2, C); o += 2 * C
    W, U = [], []
    for _ in range(L):
        W.append(p[o:o + 2 * C * C].reshape(2, C, C)); o += 2 * C * C
        U.append(p[o:o + 2 * C * C].reshape(2, C, C)); o += 2 * C * C
    w_out = p[o:o + 2 * C].reshape(2, C)
    return w_in, W, U, w_out


def _agg(H, ptr, nbr):
    """inv_deg_y * sum_{j in N(y)} H_j for H (na, S, C)."""
    deg = np.diff(ptr)
    owner = np.repeat(np.arange(len(deg)), deg)
    out = np.zeros_like(H)
    np.add.at(out, owner, H[nbr])
    return out / np.maximum(deg, 1)[:, None, None] * (deg > 0)[:, None, None]


def mpnn_forward(params, x, ptr, nbr, atype):
    """x (na, S) complex -> za (na, S), plus the per-layer inputs and messages for backward."""
    w_in, W, U, w_out = unpack(params)
    t = np.asarray(atype, dtype=np.int64)
    H = x[:, :, None] * w_in[t][:, None, :]
    ins, msgs = [], []
    for l in range(L):
        m = _agg(H, ptr, nbr)
        ins.append(H); msgs.append(m)
        H = np.einsum("ysk,ykc->ysc", H, W[l][t]) + np.einsum("ysk,ykc->ysc", m, U[l][t])
    za = x + np.einsum("ysc,yc->ys", H, w_out[t])
    return za, (ins, msgs, H)


def mpnn_backward(params, x, ptr, nbr, atype, cache, dza):
    """Gradient of a real loss with dza = dL/dRe(za) + i dL/dIm(za); returns grad (NPARAMS,)."""
    w_in, W, U, w_out = unpack(params)
    t = np.asarray(atype, dtype=np.int64)
    ins, msgs, HL = cache
    g_win = np.zeros_like(w_in); g_wout = np.zeros_like(w_out)
    gW = [np.zeros_like(w) for w in W]; gU = [np.zeros_like(u) for u in U]
    for ty in (0, 1):
        sel = t == ty
        g_wout[ty] = np.einsum("ysc,ys->c", np.conj(HL[sel]), dza[sel]).real
    d = dza[:, :, None] * w_out[t][:, None, :]
    deg = np.diff(ptr)
    for l in reversed(range(L)):
        H, m = ins[l], msgs[l]
        for ty in (0, 1):
            sel = t == ty
            gW[l][ty] = np.einsum("ysk,ysc->kc", np.conj(H[sel]), d[sel]).real
            gU[l][ty] = np.einsum("ysk,ysc->kc", np.conj(m[sel]), d[sel]).real
        # message backprop: m_y = sum_{j in N(y)} H_j / deg_y, and the graph is symmetric
        dm = np.einsum("ykc,ysc->ysk", U[l][t], d) / np.maximum(deg, 1)[:, None, None]
        d = np.einsum("ykc,ysc->ysk", W[l][t], d) + _sum_nbr(dm, ptr, nbr)
    for ty in (0, 1):
        sel = t == ty
        g_win[ty] = np.einsum("ys,ysc->c", np.conj(x[sel]), d[sel]).real
    out = [g_win.ravel()]
    for l in range(L):
        out += [gW[l].ravel(), gU[l].ravel()]
    out.append(g_wout.ravel())
    return np.concatenate(out)


def _sum_nbr(H, ptr, nbr):
    deg = np.diff(ptr)
    owner = np.repeat(np.arange(len(deg)), deg)
    out = np.zeros_like(H)
    np.add.at(out, owner, H[nbr])
    return out
