"""Shared helpers of the port-mode tests: the WR-90 port face of the golden fixture, and the DOF
permutation between the reference's set-ordered surface edges and the lexicographic ones here."""
import numpy as np

from emerge_b200.mesh import TetMesh, box_tet_mesh


def guide_mesh(g):
    nodes, tets = box_tet_mesh(10, 5, 2, float(g["wg_a"]), float(g["wg_b"]), 5e-3, seed=0)
    return TetMesh(nodes, tets)


def wall_edges(m, g):
    a, b = float(g["wg_a"]), float(g["wg_b"])
    walls = np.concatenate([m.tris_on_plane(0, 0.0), m.tris_on_plane(0, a), m.tris_on_plane(1, 0.0),
                            m.tris_on_plane(1, b)])
    return m.edges[:, m.tri_to_edge[:, walls].ravel()]


def dof_permutation(g, surface):
    """p[i] = this library's DOF index of the reference's DOF i."""
    nn, nt = surface.n_nodes, surface.n_tris
    ref_e = g["wg_sm_edges"]
    key = np.minimum(ref_e[0], ref_e[1]) * nn + np.maximum(ref_e[0], ref_e[1])
    pe = np.searchsorted(surface._ekeys, key)
    assert np.array_equal(surface._ekeys[pe], key)
    ne = pe.size
    return np.concatenate([pe, ne + np.arange(nt), ne + nt + pe, 2 * ne + nt + np.arange(nt),
                           2 * ne + 2 * nt + np.arange(nn), 2 * ne + 2 * nt + nn + pe])
