"""CPU oracle for the mesh connectivity — TEST INFRASTRUCTURE ONLY.

A direct restatement of ``Mesh3D._pre_update``'s connectivity steps
(``src/emerge/_emerge/mesh3d.py:385-497``) with Python sets, sorted tuples and dict lookups, for the
small meshes of the parity tests.  Pinned against the reference's own output
(``tests/golden/mesh_conn.npz``, produced by ``tests/golden/make_golden.py``).
"""
from __future__ import annotations

from collections import defaultdict

import numpy as np

MISSING_ID = -1234                      # mesh3d.py:27

# 1-based local pairs / triples (mesh3d.py:427, :431)
_EDGE_I, _EDGE_J = (1, 1, 1, 2, 4, 3), (2, 3, 4, 3, 2, 4)
_TRI_I, _TRI_J, _TRI_K = (1, 1, 1, 2), (2, 3, 4, 3), (3, 4, 2, 4)


def connectivity(nodes: np.ndarray, tets: np.ndarray) -> dict:
    """Return edges, tris, tet_to_edge, tet_to_tri, tri_to_tet, tri_to_edge, edge_lengths."""
    nt = tets.shape[1]
    edgeset, triset = set(), set()
    for it in range(nt):                                        # mesh3d.py:386-399
        i1, i2, i3, i4 = sorted(int(v) for v in tets[:, it])
        edgeset.update({(i1, i2), (i1, i3), (i1, i4), (i2, i3), (i2, i4), (i3, i4)})
        triset.update({(i1, i2, i3), (i1, i2, i4), (i1, i3, i4), (i2, i3, i4)})
    edges = np.array(sorted(edgeset), dtype=np.int64).T        # mesh3d.py:405-406
    tris = np.array(sorted(triset), dtype=np.int64).T
    inv_e = {tuple(int(x) for x in edges[:, i]): i for i in range(edges.shape[1])}
    inv_t = {tuple(int(x) for x in tris[:, i]): i for i in range(tris.shape[1])}

    def edge(a, b):
        return inv_e[tuple(sorted((int(a), int(b))))]

    def tri(a, b, c):
        return inv_t[tuple(sorted((int(a), int(b), int(c))))]

    t2e = np.full((6, nt), MISSING_ID, dtype=np.int64)
    t2t = np.full((4, nt), MISSING_ID, dtype=np.int64)
    tri_tets = defaultdict(list)
    for it in range(nt):                                        # mesh3d.py:424-447
        T = tets[:, it]
        t2e[:, it] = [edge(T[i - 1], T[j - 1]) for i, j in zip(_EDGE_I, _EDGE_J)]
        t2t[:, it] = [tri(T[i - 1], T[j - 1], T[k - 1]) for i, j, k in zip(_TRI_I, _TRI_J, _TRI_K)]
        for f in range(4):
            tri_tets[int(t2t[f, it])].append(it)
    tri_to_tet = np.full((2, tris.shape[1]), MISSING_ID, dtype=np.int64)
    for i in range(tris.shape[1]):
        lst = tri_tets[i]
        tri_to_tet[:len(lst), i] = lst
    tri_to_edge = np.empty((3, tris.shape[1]), dtype=np.int64)
    for i in range(tris.shape[1]):                              # mesh3d.py:474-481
        i1, i2, i3 = tris[:, i]
        tri_to_edge[:, i] = [edge(i1, i2), edge(i2, i3), edge(i1, i3)]
    d = nodes[:, edges[0]] - nodes[:, edges[1]]                 # mesh3d.py:497
    return dict(edges=edges, tris=tris, tet_to_edge=t2e, tet_to_tri=t2t, tri_to_tet=tri_to_tet,
                tri_to_edge=tri_to_edge, edge_lengths=np.sqrt(np.sum(d ** 2, axis=0)))
