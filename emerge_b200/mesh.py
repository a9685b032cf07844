"""Tetrahedral mesh connectivity in EMerge's conventions, plus a seeded box generator.

The hot path consumes a mesh exactly as EMerge's ``Mesh3D._pre_update`` lays it out
(``src/emerge/_emerge/mesh3d.py:387-497``):

* ``edges`` (2, N_e): the unique sorted ``(min, max)`` node pairs, in lexicographic order
  (``mesh3d.py:395-405``);
* ``tris`` (3, N_f): the unique sorted node triples, in lexicographic order (``mesh3d.py:406``);
* ``tet_to_edge`` (6, N_t): local vertex pairs (1,2),(1,3),(1,4),(2,3),(4,2),(3,4), 1-based in the
  tet's own vertex order (``mesh3d.py:427``);
* ``tet_to_tri`` (4, N_t): local triples (1,2,3),(1,3,4),(1,4,2),(2,3,4) (``mesh3d.py:431``);
* ``tri_to_edge`` (3, N_f): (i1,i2),(i2,i3),(i1,i3) of the sorted triple (``mesh3d.py:476-480``);
* ``tri_to_tet`` (2, N_f): tets in order of first appearance, padded with -1234 (``mesh3d.py:27,437-447``);
* ``edge_lengths`` (N_e,): Euclidean lengths (``mesh3d.py:497``).

gmsh is not part of this package. :func:`box_tet_mesh` builds the synthetic meshes used by the
tests and the benchmark: an n_x × n_y × n_z hex grid over [0,a]×[0,b]×[0,l], each hex cut into six
tets that share the (0,0,0)→(1,1,1) diagonal (so the mesh is conforming), interior nodes jittered
uniformly by up to ``jitter`` × cell size per axis from a seed, boundary nodes left on the walls.
Everything is vectorised numpy, so a 1.5 M-tet box builds in seconds.
"""
from __future__ import annotations

import itertools

import numpy as np

MISSING_ID = -1234          # Mesh3D's _MISSING_ID (mesh3d.py:27)

# local vertex pairs / triples, 0-based, in the order Mesh3D uses
TET_EDGE_PAIRS = ((0, 1), (0, 2), (0, 3), (1, 2), (3, 1), (2, 3))
TET_FACE_TRIPLES = ((0, 1, 2), (0, 2, 3), (0, 3, 1), (1, 2, 3))


def box_tet_mesh(nx: int, ny: int, nz: int, a: float, b: float, l: float,
                 jitter: float = 0.1, seed: int = 0,
                 shuffle_local: bool = False) -> tuple[np.ndarray, np.ndarray]:
    """Seeded hex→6-tet box mesh.

    Returns ``nodes`` (3, N_n) float64 and ``tets`` (4, N_t) int64.  Node id is
    ``i + (nx+1)*(j + (ny+1)*k)``; tets are emitted cell by cell (i fastest), six per cell.
    ``shuffle_local`` permutes each tet's four vertices (seeded), which exercises every local
    edge/face orientation that a gmsh mesh can produce.
    """
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, a, nx + 1)
    ys = np.linspace(0.0, b, ny + 1)
    zs = np.linspace(0.0, l, nz + 1)
    K, J, I = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    I = I.ravel(); J = J.ravel(); K = K.ravel()
    nodes = np.stack([xs[I], ys[J], zs[K]]).astype(np.float64)
    interior = (I > 0) & (I < nx) & (J > 0) & (J < ny) & (K > 0) & (K < nz)
    h = np.array([a / nx, b / ny, l / nz])
    if jitter > 0:
        nodes[:, interior] += rng.uniform(-1.0, 1.0, (3, int(interior.sum()))) * jitter * h[:, None]

    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    # cell order: i fastest, then j, then k
    ci = ci.transpose(2, 1, 0).ravel(); cj = cj.transpose(2, 1, 0).ravel(); ck = ck.transpose(2, 1, 0).ravel()

    def nid(di, dj, dk):
        return (ci + di) + (nx + 1) * ((cj + dj) + (ny + 1) * (ck + dk))

    cells = []
    for perm in itertools.permutations(range(3)):
        step = [0, 0, 0]
        path = [nid(0, 0, 0)]
        for ax in perm:
            step[ax] = 1
            path.append(nid(*step))
        cells.append(np.stack(path))              # (4, n_cells)
    tets = np.stack(cells, axis=2).reshape(4, -1).astype(np.int64)  # (4, n_cells*6), 6 per cell
    if shuffle_local:
        order = np.argsort(rng.random((4, tets.shape[1])), axis=0)
        tets = np.take_along_axis(tets, order, axis=0)
    # gmsh emits positively oriented tets; EMerge's field interpolation relies on it
    # (``elements/ned2_interp.py:220-241`` divides by |V|³), so swap two vertices where needed.
    neg = signed_volumes(nodes, tets) < 0
    tets[2, neg], tets[3, neg] = tets[3, neg].copy(), tets[2, neg].copy()
    return nodes, np.ascontiguousarray(tets)


def signed_volumes(nodes: np.ndarray, tets: np.ndarray) -> np.ndarray:
    """det[v2-v1, v3-v1, v4-v1] / 6 per tet (positive for a right-handed vertex order)."""
    p = [nodes[:, tets[i]] for i in range(4)]
    u, v, w = p[1] - p[0], p[2] - p[0], p[3] - p[0]
    return np.einsum("ij,ij->j", u, np.cross(v, w, axis=0)) / 6.0


class TetMesh:
    """Mesh connectivity with the attribute names and layouts of EMerge's ``Mesh3D``."""

    def __init__(self, nodes: np.ndarray, tets: np.ndarray):
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.tets = np.ascontiguousarray(tets, dtype=np.int64)
        nn = self.nodes.shape[1]
        T = self.tets
        srt = np.sort(T, axis=0)

        ekeys = np.concatenate([srt[p] * nn + srt[q] for p, q in
                                ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))])
        ekeys = np.unique(ekeys)
        self.edges = np.stack([ekeys // nn, ekeys % nn]).astype(np.int64)
        tkeys = np.concatenate([(srt[p] * nn + srt[q]) * nn + srt[r] for p, q, r in
                                ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))])
        tkeys = np.unique(tkeys)
        self.tris = np.stack([tkeys // (nn * nn), (tkeys // nn) % nn, tkeys % nn]).astype(np.int64)

        def edge_id(i, j):
            lo = np.minimum(i, j); hi = np.maximum(i, j)
            return np.searchsorted(ekeys, lo * nn + hi)

        def tri_id(i, j, k):
            q = np.sort(np.stack([i, j, k]), axis=0)
            return np.searchsorted(tkeys, (q[0] * nn + q[1]) * nn + q[2])

        self.tet_to_edge = np.stack([edge_id(T[p], T[q]) for p, q in TET_EDGE_PAIRS]).astype(np.int64)
        self.tet_to_tri = np.stack([tri_id(T[p], T[q], T[r]) for p, q, r in TET_FACE_TRIPLES]).astype(np.int64)
        tr = self.tris
        self.tri_to_edge = np.stack([edge_id(tr[0], tr[1]), edge_id(tr[1], tr[2]),
                                     edge_id(tr[0], tr[2])]).astype(np.int64)
        d = self.nodes[:, self.edges[0]] - self.nodes[:, self.edges[1]]
        self.edge_lengths = np.sqrt(np.sum(d ** 2, axis=0))

        # tri_to_tet: tets in ascending order of the (tet, local face) scan, as Mesh3D appends them
        nt = T.shape[1]
        flat = self.tet_to_tri.T.ravel()                       # order: tet-major, local face minor
        owner = np.repeat(np.arange(nt, dtype=np.int64), 4)
        order = np.argsort(flat, kind="stable")
        f_sorted = flat[order]
        first = np.ones(len(f_sorted), dtype=bool)
        first[1:] = f_sorted[1:] != f_sorted[:-1]
        slot = np.arange(len(f_sorted)) - np.maximum.accumulate(np.where(first, np.arange(len(f_sorted)), 0))
        self.tri_to_tet = np.full((2, self.tris.shape[1]), MISSING_ID, dtype=np.int64)
        keep = slot < 2
        self.tri_to_tet[slot[keep], f_sorted[keep]] = owner[order][keep]

    @property
    def n_nodes(self) -> int:
        return self.nodes.shape[1]

    @property
    def n_tets(self) -> int:
        return self.tets.shape[1]

    @property
    def n_edges(self) -> int:
        return self.edges.shape[1]

    @property
    def n_tris(self) -> int:
        return self.tris.shape[1]

    def tris_on_plane(self, axis: int, value: float, tol: float = 1e-12) -> np.ndarray:
        """Indices of triangles whose three vertices lie on the plane ``x[axis] == value``."""
        P = self.nodes[axis][self.tris]
        return np.where(np.all(np.abs(P - value) <= tol * max(1.0, abs(value)) + 1e-15, axis=0))[0].astype(np.int64)

    def tri_centers(self) -> np.ndarray:
        n = self.nodes
        return (n[:, self.tris[0]] + n[:, self.tris[1]] + n[:, self.tris[2]]) / 3

    def face_tets(self, tri_ids: np.ndarray) -> np.ndarray:
        """Tets sharing a node with any of the given triangles (``Mesh3D.get_face_tets``, mesh3d.py:267-272)."""
        nodes = np.unique(self.tris[:, tri_ids])
        hit = np.isin(self.tets, nodes).any(axis=0)
        return np.where(hit)[0].astype(np.int64)
