"""The precision workload's family (substrate box with a PEC strip, lumped ports and absorbing end
faces), downsized so the reference's direct solve runs in seconds: FP64 and mixed-precision sweep
solutions against SuperLU on the oracle's matrix, frequency by frequency.

On this family the FP32 inner solves stall near a relative residual of 1e-3, so the mixed-precision
request reaches 1e-8 through the fallback chain (FP64 aux-space, then FP64 block Jacobi); below about
2 GHz the aux-space correction diverges and plain block Jacobi stalls, so the frequencies here are
those where the FP64 aux-space solve converges."""
import numpy as np
import pytest

import oracle
from emerge_b200 import problems
from emerge_b200.assembler import Assembler
from emerge_b200.ports import k0_of
from emerge_b200.sweep import FrequencySweep

pytestmark = pytest.mark.gpu


def _direct(P, f):
    from oracle import abc2 as oabc2
    k0 = k0_of(f)
    E, B = oracle.tet_mass_stiffness_matrices(P.field, P.er, P.ur)
    K = (E - B * k0 ** 2).tocsr()
    Bm = P.field.empty_tri_matrix()
    pvs = []
    for p in P.ports:
        Bm, bp = oracle.assemble_robin_bc_excited(P.field, Bm, p.tri_ids, lambda x, y, z, p=p: p.get_Uinc(x, y, z, k0),
                                                  p.get_gamma(k0), oracle.dunavant4())
        pvs.append(bp)
    for bc in P.robin:
        Bm = oracle.assemble_robin_bc(P.field, Bm, bc.tri_ids, bc.get_gamma(k0))
        Bm = Bm + oabc2.abc_order_2_matrix(P.field, bc.tri_ids, bc.get_gamma2(k0))
    K = K + P.field.generate_csr(Bm)
    return K, oracle.solve_routine(K, pvs, P.solve_ids)


def test_substrate_box_fp64_and_mixed_vs_direct(cuda):
    P = problems.substrate_box(10, 8, 10)
    assert len(P.ports) == 2 and all(len(p.tri_ids) for p in P.ports)
    sw = FrequencySweep(P)
    freqs = [4.5e9, 8e9]
    systems = [(f, q) for f in freqs for q in range(2)]
    r64 = sw.solve(systems, tol=1e-12, maxit=80000, precond="aux", fallback=True)
    assert (r64.status == 0).all(), (r64.status, r64.iters, r64.relres)
    rmx = sw.solve(systems, tol=1e-8, maxit=40000, precond="aux", precision="mixed", fallback=True)
    assert (rmx.status == 0).all() and (rmx.relres <= 1e-8).all(), (rmx.status, rmx.relres)
    x64, xmx = r64.x.cpu().numpy(), rmx.x.cpu().numpy()
    for i, f in enumerate(freqs):
        K, xs = _direct(P, f)
        if i == 0:
            job = Assembler().assemble_freq_matrix(P.field, P.er, P.ur, P.ports, P.pec_tris, f, robin_bcs=P.robin)
            d = (job.A - K).tocsr()
            assert (abs(d).max() if d.nnz else 0.0) <= 1e-12 * abs(K).max()
        for q in range(2):
            ref = xs[q]
            e64 = np.linalg.norm(x64[:, 2 * i + q] - ref) / np.linalg.norm(ref)
            emx = np.linalg.norm(xmx[:, 2 * i + q] - ref) / np.linalg.norm(ref)
            assert e64 <= 1e-10, (f, q, e64)
            assert emx <= 1e-5, (f, q, emx)
    # the lumped-port S-parameters of both precisions agree
    S64, Smx = sw.sparams(r64), sw.sparams(rmx)
    for f in freqs:
        assert np.abs(S64[f] - Smx[f]).max() <= 1e-5
        assert np.all(np.abs(S64[f]) <= 1.0 + 1e-6)
