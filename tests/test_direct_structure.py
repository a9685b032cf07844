"""Host logic of the device direct solver: the nested-dissection tree and the front structure
(emerge_b200.direct) checked by a complex128 multifrontal factorization in numpy over exactly the
arrays the device receives, against SciPy's sparse direct solve."""
import numpy as np
import scipy.sparse.linalg as spl

import oracle
from emerge_b200 import problems
from emerge_b200.direct import front_structure, nested_dissection
from emerge_b200.ports import k0_of


def _system(P, f):
    fld = P.field
    E, B = oracle.tet_mass_stiffness_matrices(fld, P.er, P.ur)
    k0 = k0_of(f)
    Bm = fld.empty_tri_matrix()
    for p in P.ports:
        Bm = oracle.assemble_robin_bc(fld, Bm, p.tri_ids, p.get_gamma(k0))
    K = (E - B * k0 ** 2 + fld.generate_csr(Bm)).tocsr()
    Kp = E.copy().tocsr()
    Kp.data[:] = 0
    Kp = (Kp + K).tocsr()                # the values on E's pattern (the device plan's pattern)
    Kp.sort_indices()
    return Kp


def _tree(P, leaf):
    m, fld = P.mesh, P.field
    H = m.n_edges + m.n_tris
    free = np.ones(2 * H, bool)
    free[P.pec_ids] = False
    cen = m.nodes[:, m.tets].mean(axis=1)
    return nested_dissection(fld.tet_to_field[:10], H, cen, free, H, leaf_tets=leaf), free


def _multifrontal_solve(S, vals, rhs):
    """Unpivoted-across-fronts LU with partial pivoting inside each front's own block (complex128)."""
    upd, facts = {}, {}
    for v in np.argsort(S.level, kind="stable"):
        e, b = int(S.e[v]), int(S.b[v])
        n = e + b
        F = np.zeros(n * n, dtype=np.complex128)
        a0, a1 = S.asm_ptr[v], S.asm_ptr[v + 1]
        F[S.asm_off[a0:a1]] = vals[S.asm_slot[a0:a1]]
        F = F.reshape(n, n, order="F")
        for c in np.flatnonzero(S.parent == v):
            mp = S.ea[S.ea_ptr[c]:S.ea_ptr[c] + S.b[c]]
            F[np.ix_(mp, mp)] += upd.pop(c)
        import scipy.linalg as sla
        lu, piv = sla.lu_factor(F[:e, :e]) if e else (np.zeros((0, 0)), np.zeros(0, int))
        L21 = sla.solve_triangular(lu, F[e:, :e].T, trans=1, lower=False).T if e else np.zeros((b, 0))
        Fp = F[:e, e:].copy()
        for j, r in enumerate(piv):
            Fp[[j, r]] = Fp[[r, j]]
        U12 = sla.solve_triangular(lu, Fp, lower=True, unit_diagonal=True) if e else np.zeros((0, b))
        upd[v] = F[e:, e:] - L21 @ U12
        facts[v] = (lu, piv, L21, U12)
    y, uvec = {}, {}
    for v in np.argsort(S.level, kind="stable"):
        e, b = int(S.e[v]), int(S.b[v])
        d = S.fdof[S.fdof_ptr[v]:S.fdof_ptr[v + 1]]
        w = np.zeros(e + b, dtype=np.complex128)
        w[:e] = rhs[d[:e]]
        for c in np.flatnonzero(S.parent == v):
            w[S.ea[S.ea_ptr[c]:S.ea_ptr[c] + S.b[c]]] += uvec.pop(c)
        lu, piv, L21, U12 = facts[v]
        wo = w[:e].copy()
        for j, r in enumerate(piv):
            wo[[j, r]] = wo[[r, j]]
        import scipy.linalg as sla
        yo = sla.solve_triangular(lu, wo, lower=True, unit_diagonal=True) if e else wo
        y[v] = yo
        uvec[v] = w[e:] - L21 @ yo
    x = np.zeros(S.n, dtype=np.complex128)
    for v in np.argsort(S.level, kind="stable")[::-1]:
        e = int(S.e[v])
        d = S.fdof[S.fdof_ptr[v]:S.fdof_ptr[v + 1]]
        lu, piv, L21, U12 = facts[v]
        import scipy.linalg as sla
        if e:
            x[d[:e]] = sla.solve_triangular(lu, y[v] - U12 @ x[d[e:]], lower=False)
    return x


def test_tree_covers_every_free_dof_once_and_boundaries_are_ancestors():
    P = problems.waveguide(nx=5, ny=3, nz=8)
    T, free = _tree(P, 24)
    assert np.array_equal(np.sort(T.perm), np.flatnonzero(free))
    assert (T.pos[free] >= 0).all() and (T.pos[~free] == -1).all()
    # postorder: parents after children, one root, every boundary DOF eliminated by an ancestor
    assert (T.parent[:-1] > np.arange(T.n_nodes - 1)).all() and T.parent[-1] == -1
    node_of_pos = np.repeat(np.arange(T.n_nodes), T.own_size())
    for v in range(T.n_nodes):
        bd = T.bnd[T.bnd_ptr[v]:T.bnd_ptr[v + 1]]
        owners = node_of_pos[T.pos[bd]]
        anc, a = set(), T.parent[v]
        while a >= 0:
            anc.add(int(a))
            a = T.parent[a]
        assert set(owners.tolist()) <= anc
        assert (np.diff(T.pos[bd]) > 0).all()


def test_multifrontal_over_the_front_structure_matches_scipy():
    P = problems.waveguide(nx=6, ny=3, nz=10)
    K = _system(P, 10e9)
    T, free = _tree(P, 32)
    S = front_structure(T, K.indptr, K.indices)
    ids = P.solve_ids
    # every CSR entry of the free block is assembled exactly once
    rows = np.repeat(np.arange(K.shape[0]), np.diff(K.indptr))
    nfree = int((free[rows] & free[K.indices]).sum())
    assert S.asm_ptr[-1] == nfree == len(np.unique(S.asm_slot))
    rng = np.random.default_rng(1)
    b = np.zeros(K.shape[0], complex)
    b[ids] = rng.standard_normal(len(ids)) + 1j * rng.standard_normal(len(ids))
    x = _multifrontal_solve(S, K.data, b)
    xr = np.zeros_like(b)
    xr[ids] = spl.spsolve(K[ids][:, ids].tocsc(), b[ids])
    assert np.linalg.norm(x - xr) <= 1e-11 * np.linalg.norm(xr)
    assert np.abs(x[~free]).max() == 0


def test_equilibrated_multifrontal_matches_scipy_at_low_frequency():
    """The device factors D^-1/2 K D^-1/2 (D = |diag K|_1, the scale of each DOF taken from its own
    diagonal) and returns D^-1/2 (LU)^-1 D^-1/2 b: the same algebra in complex128 over the same front
    structure reproduces SciPy's solve, here at a low frequency where the gradient-type DOFs' diagonals
    are far below the curl-curl scale."""
    P = problems.substrate_box(8, 6, 6)
    K = _system(P, 1e9)
    T, free = _tree(P, 32)
    S = front_structure(T, K.indptr, K.indices)
    ids = P.solve_ids
    d = K.diagonal()
    a = np.abs(d.real) + np.abs(d.imag)
    assert a[ids].min() < 0.1 * a[ids].max()         # the spread the equilibration removes (grows as h shrinks)
    sc = np.where(a > 0, 1.0 / np.sqrt(np.where(a > 0, a, 1.0)), 1.0)
    rows = np.repeat(np.arange(K.shape[0]), np.diff(K.indptr))
    vals = K.data * sc[rows] * sc[K.indices]
    ks = vals[K.indptr[:-1] + np.array([np.searchsorted(K.indices[K.indptr[r]:K.indptr[r + 1]], r)
                                        for r in range(K.shape[0])])]
    assert np.allclose(np.abs(ks.real) + np.abs(ks.imag), 1.0)   # unit diagonal after scaling
    rng = np.random.default_rng(2)
    b = np.zeros(K.shape[0], complex)
    b[ids] = rng.standard_normal(len(ids)) + 1j * rng.standard_normal(len(ids))
    x = sc * _multifrontal_solve(S, vals, sc * b)
    xr = np.zeros_like(b)
    xr[ids] = spl.spsolve(K[ids][:, ids].tocsc(), b[ids])
    assert np.linalg.norm(x[ids] - xr[ids]) <= 1e-10 * np.linalg.norm(xr[ids])
