"""GPU auxiliary space (emfem_aux_*) and the preconditioner network (emfem_mpnn_*): the discrete
gradient against the oracle's fit of the reference basis, the aux operator diagonals against SciPy,
network gradients against the float64 oracle, the aux-preconditioned solve against the reference's
SuperLU solution, and what training gains."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from oracle import auxspace as oa
from emerge_b200 import problems
from emerge_b200.auxspace import AuxSpace, Network, make_pairs, train
from emerge_b200.mesh import TetMesh, box_tet_mesh
from emerge_b200.nedelec2 import Nedelec2
from emerge_b200.sweep import FrequencySweep

pytestmark = pytest.mark.gpu


def _G_from_export(ex, n, na):
    gcol = ex["gcol"].cpu().numpy(); gval = ex["gval"].cpu().numpy()
    r = np.repeat(np.arange(n), 6)
    keep = gcol.ravel() >= 0
    return sp.csr_matrix((gval.ravel()[keep], (r[keep], gcol.ravel()[keep])), shape=(n, na))


def test_discrete_gradient_vs_oracle_fit(cuda):
    nodes, tets = box_tet_mesh(4, 3, 3, 1.0e-2, 0.8e-2, 1.1e-2, jitter=0.15, seed=5, shuffle_local=True)
    m = TetMesh(nodes, tets)
    f = Nedelec2(m)
    aux = AuxSpace(m)
    ex = aux.export()
    G = _G_from_export(ex, f.n_field, aux.n_aux)
    Go = oa.gradient_matrix(m, f)
    assert abs(G - Go).max() <= 1e-9 * abs(Go).max()
    # G^T export is the exact transpose with sorted rows
    GT = sp.csr_matrix((ex["gt_val"].cpu().numpy(), ex["gt_row"].cpu().numpy(), ex["gt_ptr"].cpu().numpy()),
                       shape=(aux.n_aux, f.n_field))
    assert abs(GT - G.T).max() == 0
    # incidence graph: vertex -> incident edges, edge -> its two vertices, symmetric
    ptr, nbr = ex["graph_ptr"].cpu().numpy(), ex["graph_nbr"].cpu().numpy()
    A = sp.csr_matrix((np.ones(len(nbr)), nbr, ptr), shape=(aux.n_aux, aux.n_aux))
    assert abs(A - A.T).max() == 0
    e0 = m.n_nodes + 7
    assert sorted(nbr[ptr[e0]:ptr[e0 + 1]]) == sorted(m.edges[:, 7].tolist())


@pytest.fixture(scope="module")
def guide(cuda):
    P = problems.waveguide()
    sw = FrequencySweep(P)
    return P, sw


def test_aux_diagonals_vs_scipy(guide):
    P, sw = guide
    aux = sw.aux_space()
    ex = aux.export()
    G = _G_from_export(ex, sw.n, aux.n_aux)
    ip, ix = sw.plan.host_pattern()
    E = sp.csr_matrix((sw.E.cpu().numpy(), ix, ip), shape=(sw.n, sw.n))
    B = sp.csr_matrix((sw.B.cpu().numpy(), ix, ip), shape=(sw.n, sw.n))
    diag = aux.set_operator(sw).cpu().numpy().reshape(2 + sw.n_ports, aux.n_aux)
    dB = oa.aux_diagonals(G, B)
    assert np.abs(diag[1] - dB).max() <= 1e-12 * np.abs(dB).max()
    assert np.abs(diag[0]).max() <= 1e-10 * np.abs(oa.aux_diagonals(G, abs(E))).max()   # curl grad = 0
    # Robin patch of port 0 against SciPy
    pr = sw.patch_rows.cpu().numpy(); pp = sw.patch_rowptr.cpu().numpy()
    pc = sw.patch_cols.cpu().numpy(); pv = sw.patch_vals.cpu().numpy(); po = sw.patch_port.cpu().numpy()
    rows = np.repeat(pr, np.diff(pp))
    for q in range(sw.n_ports):
        sel = po == q
        R = sp.csr_matrix((pv[sel], (rows[sel], pc[sel])), shape=(sw.n, sw.n))
        dR = oa.aux_diagonals(G, R)
        assert np.abs(diag[2 + q] - dR).max() <= 1e-12 * np.abs(dR).max()
    # usable aux nodes: support entirely on free DOFs
    mask = aux.mask.cpu().numpy().astype(bool)
    free = sw.mask.cpu().numpy().astype(bool)
    expect = np.array([free[G.T.getrow(y).indices].all() and G.T.getrow(y).nnz > 0 for y in range(aux.n_aux)])
    assert np.array_equal(mask, expect)


def test_aux_preconditioned_solve_matches_superlu_golden(guide, golden):
    """BiCGStab with the aux-space correction reaches the reference's SuperLU solution, in far
    fewer iterations than block Jacobi alone."""
    P, sw = guide
    g = golden("config1")
    f = float(g["f"])
    res = sw.solve([(f, 0), (f, 1)], tol=1e-12, maxit=20000, precond="aux")
    assert (res.status == 0).all(), (res.status, res.iters, res.relres)
    x = res.x.cpu().numpy()
    for j, key in enumerate(("x1", "x2")):
        gx = g[key]
        assert np.linalg.norm(x[:, j] - gx) / np.linalg.norm(gx) <= 1e-10
    bj = sw.solve([(f, 0), (f, 1)], tol=1e-8, maxit=20000, precond="block_jacobi")
    ax = sw.solve([(f, 0), (f, 1)], tol=1e-8, maxit=20000, precond="aux")
    assert ax.iters.max() * 4 < bj.iters.max(), (ax.iters, bj.iters)
    mx = sw.solve([(f, 0), (f, 1)], tol=1e-8, maxit=20000, precond="aux", precision="mixed")
    assert (mx.status == 0).all() and (mx.relres <= 1e-8).all(), (mx.status, mx.iters, mx.relres)


def test_network_forward_backward_vs_oracle(guide):
    P, sw = guide
    aux = sw.aux_space()
    ex = aux.export()
    ptr, nbr = ex["graph_ptr"].cpu().numpy(), ex["graph_nbr"].cpu().numpy()
    atype = (np.arange(aux.n_aux) >= P.mesh.n_nodes).astype(np.uint8)
    net = Network(aux, seed=3, init="random")
    rng = np.random.default_rng(1)
    S = 3
    x = (rng.standard_normal((aux.n_aux, S)) + 1j * rng.standard_normal((aux.n_aux, S))).astype(np.complex64)
    tgt = (rng.standard_normal((aux.n_aux, S)) + 1j * rng.standard_normal((aux.n_aux, S)))
    za = net.forward(torch.from_numpy(x).to(aux.device)).cpu().numpy()
    p = net.params.cpu().numpy().astype(np.float64)
    zo, cache = oa.mpnn_forward(p, x.astype(np.complex128), ptr, nbr, atype)
    assert np.abs(za - zo).max() <= 2e-5 * np.abs(zo).max()
    dza = 2 * (zo - tgt)
    grad = net.backward(torch.from_numpy(dza.astype(np.complex64)).to(aux.device)).cpu().numpy()
    go = oa.mpnn_backward(p, x.astype(np.complex128), ptr, nbr, atype, cache, dza)
    scale = np.abs(go).max()
    assert np.abs(grad - go).max() <= 1e-4 * scale, np.abs(grad - go).max() / scale
    # every parameter block receives its gradient (w_in, W/U of each layer, w_out)
    assert np.abs(grad[:64]).max() > 0 and np.abs(grad[-64:]).max() > 0
    # the tensor-core inference form used inside the solve (TF32 inputs): same network, looser bound
    zt = net.infer(torch.from_numpy(x).to(aux.device)).cpu().numpy()
    assert np.abs(zt - zo).max() <= 5e-3 * np.abs(zo).max(), np.abs(zt - zo).max() / np.abs(zo).max()
    # S a multiple of 8 takes the one-node-per-tile gather of the inference kernel
    x16 = (rng.standard_normal((aux.n_aux, 16)) + 1j * rng.standard_normal((aux.n_aux, 16))).astype(np.complex64)
    z16 = net.infer(torch.from_numpy(x16).to(aux.device)).cpu().numpy()
    zo16, _ = oa.mpnn_forward(p, x16.astype(np.complex128), ptr, nbr, atype)
    assert np.abs(z16 - zo16).max() <= 5e-3 * np.abs(zo16).max(), np.abs(z16 - zo16).max() / np.abs(zo16).max()
    # each column depends on its own input column only: the row-by-row gather (S = 3) agrees
    z3 = net.infer(torch.from_numpy(x16[:, :3].copy()).to(aux.device)).cpu().numpy()
    assert np.abs(z3 - z16[:, :3]).max() <= 1e-6 * np.abs(z16).max()


def test_training_reduces_correction_loss_and_learned_solve_converges(guide, golden):
    P, sw = guide
    aux = sw.aux_space()
    train_sys = [(f, q) for f in np.linspace(8.125e9, 11.875e9, 9) for q in (0, 1)]
    pairs = make_pairs(sw, train_sys, snapshots=(4, 16, 48, 128))
    held = make_pairs(sw, [(10.5e9, 0)], snapshots=(16, 64))
    net = Network(aux, seed=0)
    rep = train(net, sw, pairs, heldout=held, steps=300, batch=8, lr=2e-3, validate=[(9.3e9, 0), (9.3e9, 1)])
    assert rep.loss_last < rep.loss_first
    # the training objective generalises to held-out pairs ...
    assert rep.loss_learned_heldout < rep.loss_jacobi_heldout, rep
    # ... and validation keeps the solve no slower than the aux Jacobi the network started from
    assert rep.validation_iters_aux > 0 and rep.validation_iters_learned > 0
    if not rep.accepted:
        assert float(net.params[-64:].abs().max()) == 0.0
    sw.set_network(net)
    g = golden("config1")
    f = float(g["f"])
    res = sw.solve([(f, 0), (f, 1)], tol=1e-10, maxit=20000, precond="learned")
    assert (res.status == 0).all(), (res.status, res.iters, res.relres)
    x = res.x.cpu().numpy()
    for j, key in enumerate(("x1", "x2")):
        gx = g[key]
        assert np.linalg.norm(x[:, j] - gx) / np.linalg.norm(gx) <= 1e-8
    # what the trained network gains over the method without it: the aux-space Jacobi (the same
    # preconditioner with the network's output weights at zero), on systems outside the training and
    # validation sets.  Validation only keeps a learned term that beat the aux Jacobi; when it rejected
    # the term, precond="learned" is the aux Jacobi exactly and the gain is zero.
    held_sys = [(10.5e9, 0), (10.5e9, 1)]
    aux_j = sw.solve(held_sys, tol=1e-8, maxit=40000, precond="aux")
    learned = sw.solve(held_sys, tol=1e-8, maxit=40000, precond="learned", fallback=True)
    assert (aux_j.status == 0).all() and (learned.status == 0).all()
    assert learned.fallbacks == 0
    if rep.accepted:
        assert learned.iters.sum() <= 1.25 * aux_j.iters.sum(), (learned.iters, aux_j.iters)
    else:
        assert (learned.iters == aux_j.iters).all(), (learned.iters, aux_j.iters)
        assert torch.equal(learned.x, aux_j.x)
    # and both far below plain block Jacobi: the aux-space structure, not the network, carries that
    plain = sw.solve(held_sys, tol=1e-8, maxit=40000, precond="block_jacobi")
    assert (plain.status == 0).all()
    assert aux_j.iters.max() * 4 < plain.iters.max(), (aux_j.iters, plain.iters)
    sw.set_network(None)
