"""Parity at the benchmarked sizes: the fused device assembly of the full 384 000-tet cavity (the
bench workload) and of a config-3-style box with anisotropic diagonal mu_r against the oracle's
restatement of the reference's _matrix_builder + coo_matrix(...).tocsr() (ASM/curlcurl.py:145-173,
:419-466): CSR pattern bit-exact, every value within 1e-12 of its row's largest entry, and per-element
matrices of a random sample of tets within 1e-12 relative Frobenius."""
import gc
import os

import numpy as np
import pytest

import oracle
from conftest import rel_fro_per_row
from emerge_b200 import assembly, problems
from emerge_b200.mesh import TetMesh, box_tet_mesh
from emerge_b200.nedelec2 import Nedelec2

pytestmark = pytest.mark.gpu


def _compare_csr(X, Xo):
    """(max over rows of the relative Frobenius error, max entry error relative to its row's largest entry).
    A CSR value sums up to ~14 element contributions that partly cancel, so its error is bounded by the
    elements' (each <= 1e-12 relative) rather than by the row's own largest entry."""
    assert np.array_equal(X.indptr, Xo.indptr) and np.array_equal(X.indices, Xo.indices)
    rows = np.repeat(np.arange(X.shape[0]), np.diff(X.indptr))
    d = np.abs(X.data - Xo.data)
    rowmax = np.maximum.reduceat(np.abs(Xo.data), Xo.indptr[:-1])
    num = np.sqrt(np.add.reduceat(d * d, Xo.indptr[:-1]))
    den = np.sqrt(np.add.reduceat(np.abs(Xo.data) ** 2, Xo.indptr[:-1]))
    fro = num / np.where(den > 0, den, 1.0)
    ent = d / np.where(rowmax > 0, rowmax, 1.0)[rows]
    return float(fro.max()), float(ent.max())


def _full_parity(field, er, ur, n_sample=2000, seed=0):
    m = field.mesh
    E, B = assembly.tet_mass_stiffness_matrices(field, er, ur)
    oracle.set_threads(len(os.sched_getaffinity(0)))      # the oracle's OpenMP loop on every host core
    Eo, Bo = oracle.tet_mass_stiffness_matrices(field, er, ur)
    for X, Xo in ((E, Eo), (B, Bo)):
        fro, ent = _compare_csr(X, Xo)
        assert fro <= 1e-12 and ent <= 4e-12, (fro, ent)
    del E, Eo
    del B, Bo
    gc.collect()
    # per-element matrices of a random sample of tets through emfem_ned2_tet_matrices
    s = np.sort(np.random.default_rng(seed).choice(m.n_tets, n_sample, replace=False))
    args = (m.nodes, m.tets[:, s], m.tris, m.edges, m.edge_lengths, field.tet_to_field[:, s], m.tet_to_edge[:, s],
            ur[:, :, s], er[:, :, s])
    dE, dB, r, c = assembly._matrix_builder(*args)
    oE, oB, orr, oc = oracle.matrix_builder(*args)
    assert rel_fro_per_row(dE.reshape(-1, 400), oE.reshape(-1, 400)) <= 1e-12
    assert rel_fro_per_row(dB.reshape(-1, 400), oB.reshape(-1, 400)) <= 1e-12
    assert np.array_equal(r, orr) and np.array_equal(c, oc)


def test_cavity_384000_tets_vs_oracle(cuda):
    P = problems.cavity()
    assert P.mesh.n_tets == 384000
    _full_parity(P.field, P.er, P.ur)
    assembly.release_host_buffers(P.field)


def test_anisotropic_mu_box_vs_oracle(cuda):
    """A box of the batched-mesh family (about 150 000 tets): per-tet eps' ~ U[1,12], tan d ~ U[0,5e-3],
    diagonal mu_r ~ U[1,2] on a seeded 10 % of tets (the diagonal path of the reference's matinv)."""
    rng = np.random.default_rng(21)
    nodes, tets = box_tet_mesh(30, 28, 30, 0.02, 0.0187, 0.02, jitter=0.1, seed=33)
    m = TetMesh(nodes, tets)
    f = Nedelec2(m)
    nt = m.n_tets
    d = rng.uniform(1, 12, nt) * (1 - 1j * rng.uniform(0, 5e-3, nt))
    er = np.zeros((3, 3, nt), np.complex128)
    ur = np.zeros((3, 3, nt), np.complex128)
    aniso = rng.random(nt) < 0.1
    for c in range(3):
        er[c, c] = d
        ur[c, c] = np.where(aniso, rng.uniform(1, 2, nt), 1.0)
    assert aniso.sum() > 10000
    _full_parity(f, er, ur, seed=1)
    assembly.release_host_buffers(f)
