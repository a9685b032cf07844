"""CPU checks of the auxiliary-space oracle: the fitted discrete gradient is exact (curl-free in the
reference's own curl-curl matrix) and the network oracle's backward matches finite differences."""
import numpy as np

import oracle
from oracle import auxspace as oa
from emerge_b200.mesh import TetMesh, box_tet_mesh
from emerge_b200.nedelec2 import Nedelec2


def test_oracle_gradient_is_curl_free_and_entity_local():
    nodes, tets = box_tet_mesh(3, 2, 3, 1.0e-2, 0.8e-2, 1.1e-2, jitter=0.15, seed=3, shuffle_local=True)
    m = TetMesh(nodes, tets)
    f = Nedelec2(m)
    G = oa.gradient_matrix(m, f)
    nt = m.n_tets
    eye = np.zeros((3, 3, nt), complex)
    for i in range(3):
        eye[i, i] = 1.0
    E, B = oracle.tet_mass_stiffness_matrices(f, eye, eye)
    ratio = np.abs((E @ G).toarray()).max() / (np.abs(E.data).max() * np.abs(G.data).max())
    assert ratio < 1e-10
    # edge DOF rows touch 3 aux nodes (2 vertices + the edge), face DOF rows 6
    cnt = np.diff(G.indptr)
    H = m.n_edges + m.n_tris
    for half in (0, H):
        assert np.all(cnt[half:half + m.n_edges] == 3)
        assert np.all(cnt[half + m.n_edges:half + H] == 6)
    # gradients of the vertex hats sum to grad(1) = 0
    assert np.abs(G[:, :m.n_nodes].sum(axis=1)).max() < 1e-9 * np.abs(G.data).max()


def _graph(rng, nv, ne):
    ed = np.array([rng.choice(nv, 2, replace=False) for _ in range(ne)])
    nb = [[] for _ in range(nv + ne)]
    for e, (a, b) in enumerate(ed):
        nb[a].append(nv + e); nb[b].append(nv + e); nb[nv + e] += [a, b]
    ptr = np.concatenate([[0], np.cumsum([len(x) for x in nb])])
    return ptr, np.array([j for x in nb for j in sorted(x)]), (np.arange(nv + ne) >= nv).astype(np.uint8)


def test_network_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    ptr, nbr, atype = _graph(rng, 10, 30)
    na, S = 40, 3
    p = rng.standard_normal(oa.NPARAMS) * 0.2
    x = rng.standard_normal((na, S)) + 1j * rng.standard_normal((na, S))
    tgt = rng.standard_normal((na, S)) + 1j * rng.standard_normal((na, S))

    def loss(q):
        za, _ = oa.mpnn_forward(q, x, ptr, nbr, atype)
        return np.sum(np.abs(za - tgt) ** 2)

    za, cache = oa.mpnn_forward(p, x, ptr, nbr, atype)
    g = oa.mpnn_backward(p, x, ptr, nbr, atype, cache, 2 * (za - tgt))
    idx = np.concatenate([rng.choice(oa.NPARAMS, 40, replace=False), [0, 63, 64, oa.NPARAMS - 1, oa.NPARAMS - 40]])
    eps = 1e-6
    fd = []
    for i in idx:
        d = np.zeros(oa.NPARAMS); d[i] = eps
        fd.append((loss(p + d) - loss(p - d)) / (2 * eps))
    fd = np.array(fd)
    assert np.abs(fd - g[idx]).max() <= 1e-7 * np.abs(fd).max()
