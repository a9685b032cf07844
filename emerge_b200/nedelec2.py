"""Nédélec-2 degree-of-freedom maps (the DOF layout of the drop-in contract).

Follows ``Nedelec2.__init__`` (``src/emerge/_emerge/elements/nedelec2.py:28-66``) and the
``FEMBasis`` helpers (``src/emerge/_emerge/elements/femdata.py:105-134``):

* N = 2·N_e + 2·N_f DOFs, ordered [edge 1st-kind | face 1st-kind | edge 2nd-kind | face 2nd-kind];
* ``tet_to_field`` (20, N_t) = [tet_to_edge; tet_to_tri + N_e; tet_to_edge + N_e + N_f;
  tet_to_tri + 2·N_e + N_f];
* ``edge_to_field`` (2, N_e) and ``tri_to_field`` (8, N_f) = [3 edges, face, 3 edges + N_e + N_f,
  face + 2·N_e + N_f].

An entity (edge ``e`` or face ``f``) owns the two DOFs ``d`` and ``d + N_e + N_f`` with
``d = e`` or ``d = N_e + f``; the device kernels use that pairing throughout.
"""
from __future__ import annotations

import numpy as np
from scipy.sparse import csr_matrix


class Nedelec2:
    n_tet_dofs = 20
    n_tri_dofs = 8

    def __init__(self, mesh):
        self.mesh = mesh
        ne, nf, nt = mesh.n_edges, mesh.n_tris, mesh.n_tets
        self.n_edges, self.n_tris, self.n_tets = ne, nf, nt
        self.nedges, self.ntris, self.ntets = ne, nf, nt
        self.n_field = 2 * ne + 2 * nf
        self.nfield = self.n_field

        t2f = np.zeros((20, nt), dtype=np.int64)
        t2f[:6] = mesh.tet_to_edge
        t2f[6:10] = mesh.tet_to_tri + ne
        t2f[10:16] = mesh.tet_to_edge + (nf + ne)
        t2f[16:20] = mesh.tet_to_tri + (nf + 2 * ne)
        self.tet_to_field = t2f

        self.edge_to_field = np.stack([np.arange(ne), np.arange(ne) + nf + ne]).astype(np.int64)
        tr2f = np.zeros((8, nf), dtype=np.int64)
        tr2f[:3] = mesh.tri_to_edge
        tr2f[3] = np.arange(nf) + ne
        tr2f[4:7] = mesh.tri_to_edge + ne + nf
        tr2f[7] = np.arange(nf) + 2 * ne + nf
        self.tri_to_field = tr2f
        self._rows, self._cols = self.empty_tri_rowcol()

    # ---- FEMBasis helpers (femdata.py:88-134) ----
    def empty_tri_matrix(self) -> np.ndarray:
        return np.zeros((self.n_tris * 64,), dtype=np.complex128)

    def empty_tri_rowcol(self) -> tuple[np.ndarray, np.ndarray]:
        """Row-major 8×8 COO indices per triangle (femdata.py:105-121), vectorised."""
        idx = self.tri_to_field                                   # (8, N_f)
        rows = np.repeat(idx.T, 8, axis=1).ravel()               # row = idx[ii] for k = 8*ii + jj
        cols = np.tile(idx.T, (1, 8)).ravel()                    # col = idx[jj]
        return rows.astype(np.int64), cols.astype(np.int64)

    def generate_csr(self, data: np.ndarray) -> csr_matrix:
        """CSR of the per-triangle blocks with exact zeros dropped (femdata.py:131-134)."""
        ids = np.flatnonzero(data != 0)
        return csr_matrix((data[ids], (self._rows[ids], self._cols[ids])), shape=(self.n_field, self.n_field))

    def pec_dofs(self, tri_ids: np.ndarray) -> np.ndarray:
        """DOFs fixed by PEC on the given boundary triangles (``assembler.py:290-307``)."""
        tri_ids = np.asarray(tri_ids, dtype=np.int64)
        eids = self.mesh.tri_to_edge[:, tri_ids].ravel()
        ids = np.concatenate([self.edge_to_field[:, eids].ravel(), self.tri_to_field[:, tri_ids].ravel()])
        return np.unique(ids)

    def solve_ids(self, pec_ids: np.ndarray) -> np.ndarray:
        """All DOFs not fixed by PEC, ascending (``assembler.py:406-407``)."""
        mask = np.ones(self.n_field, dtype=bool)
        mask[np.asarray(pec_ids, dtype=np.int64)] = False
        return np.flatnonzero(mask).astype(np.int64)
