"""Host logic of the grouped multi-mesh layout (``batch.grouped_layout``) on a union built on the CPU."""
import numpy as np
import scipy.sparse as sp

import oracle
from emerge_b200.batch import grouped_layout
from emerge_b200.mesh import TetMesh, box_tet_mesh
from emerge_b200.nedelec2 import Nedelec2


def _meshes():
    out = []
    for k, (nx, ny, nz) in enumerate(((2, 2, 3), (3, 1, 2), (1, 2, 2))):
        nodes, tets = box_tet_mesh(nx, ny, nz, 1e-2, 8e-3, 1.2e-2, seed=k)
        out.append(TetMesh(nodes, tets))
    return out


def test_layout_rows_are_whole_blocks_and_keep_each_mesh_in_order():
    ms = _meshes()
    ne = [m.n_edges for m in ms]
    nf = [m.n_tris for m in ms]
    hoff, perm = grouped_layout(ne, nf, align=256)
    h = int(hoff[-1])
    assert (hoff % 256 == 0).all() and perm.size == 2 * sum(ne) + 2 * sum(nf)
    assert np.unique(perm).size == perm.size and perm.max() < 2 * h          # injective, in range
    # mesh g's local DOF d (its own numbering) lands at hoff[g] + d (first kind) / h + hoff[g] + d - H_g
    Ne, Nf = sum(ne), sum(nf)
    eo, to = np.concatenate([[0], np.cumsum(ne)]), np.concatenate([[0], np.cumsum(nf)])
    for g in range(len(ms)):
        H = ne[g] + nf[g]
        d = np.arange(2 * H)
        kind2 = d >= H
        e = d % H
        union = np.where(e < ne[g], eo[g] + e, Ne + to[g] + (e - ne[g])) + kind2 * (Ne + Nf)
        want = np.where(kind2, h + hoff[g] + e, hoff[g] + e)
        assert np.array_equal(perm[union], want)


def test_union_matrix_permuted_is_block_diagonal_with_each_mesh_unchanged():
    """The union's matrix (meshes assembled separately, placed block-diagonally in union numbering) moved
    by the layout equals each mesh's own matrix on its rows: the columns of a row keep their order."""
    ms = _meshes()
    mats, ne, nf = [], [], []
    for m in ms:
        f = Nedelec2(m)
        er = np.zeros((3, 3, m.n_tets), complex)
        for i in range(3):
            er[i, i] = 1.0 + 0.1j
        E, _ = oracle.tet_mass_stiffness_matrices(f, er, er)
        mats.append(E.tocsr()); ne.append(m.n_edges); nf.append(m.n_tris)
    hoff, perm = grouped_layout(ne, nf, align=256)
    n = 2 * int(hoff[-1])
    Ne, Nf = sum(ne), sum(nf)
    eo, to = np.concatenate([[0], np.cumsum(ne)]), np.concatenate([[0], np.cumsum(nf)])
    rows, cols, vals = [], [], []
    for g, E in enumerate(mats):
        H = ne[g] + nf[g]
        e = np.arange(2 * H) % H
        u = np.where(e < ne[g], eo[g] + e, Ne + to[g] + (e - ne[g])) + (np.arange(2 * H) >= H) * (Ne + Nf)
        C = E.tocoo()
        rows.append(u[C.row]); cols.append(u[C.col]); vals.append(C.data)
    U = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(2 * (Ne + Nf), 2 * (Ne + Nf)))
    P = sp.csr_matrix((np.ones(perm.size), (perm, np.arange(perm.size))), shape=(n, perm.size))
    Gm = (P @ U @ P.T).tocsr()
    h = n // 2
    for g, E in enumerate(mats):
        H = ne[g] + nf[g]
        loc = np.concatenate([hoff[g] + np.arange(H), h + hoff[g] + np.arange(H)])
        assert abs(Gm[loc][:, loc] - E).max() == 0
        # nothing couples mesh g to another mesh
        outside = np.setdiff1d(np.arange(n), loc)
        assert Gm[loc][:, outside].nnz == 0
