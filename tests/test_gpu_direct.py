"""The device multifrontal LU (emerge_b200.direct.DeviceLU, emfem_mf_*) and the LU-preconditioned
sweep (emfem_krylov_solve_lu) against the reference's direct solve: SuperLU on the oracle's matrices
(SolverSuperLU, src/emerge/_emerge/solver.py:535-572) and the reference's own SuperLU solutions."""
import numpy as np
import pytest
import scipy.sparse.linalg as spl
import torch

import oracle
from emerge_b200 import problems
from emerge_b200.direct import DeviceLU
from emerge_b200.ports import k0_of
from emerge_b200.sweep import FrequencySweep

pytestmark = pytest.mark.gpu


def _oracle_solutions(P, f, ports):
    """SuperLU on the oracle's K_f, one factorization for every excited port in ``ports`` (the reference
    reuses its LU across the ports of a frequency, MW/simjob.py:82-107)."""
    fld = P.field
    E, B = oracle.tet_mass_stiffness_matrices(fld, P.er, P.ur)
    k0 = k0_of(f)
    Bm = fld.empty_tri_matrix()
    bs = {}
    for i, p in enumerate(P.ports):
        Bm, bp = oracle.assemble_robin_bc_excited(fld, Bm, p.tri_ids, lambda x, y, z, p=p: p.get_Uinc(x, y, z, k0),
                                                  p.get_gamma(k0), oracle.dunavant4())
        bs[i] = bp
    K = (E - B * k0 ** 2 + fld.generate_csr(Bm)).tocsc()
    ids = P.solve_ids
    lu = spl.splu(K[ids][:, ids].tocsc())
    out = []
    for q in ports:
        x = np.zeros(fld.n_field, complex)
        x[ids] = lu.solve(bs[q][ids])
        out.append(x)
    return out, K, lu


def _oracle_solution(P, f, q):
    """SuperLU on the oracle's K_f with port q's excitation (the reference's SolveRoutine path)."""
    fld = P.field
    E, B = oracle.tet_mass_stiffness_matrices(fld, P.er, P.ur)
    k0 = k0_of(f)
    Bm = fld.empty_tri_matrix()
    b = np.zeros(fld.n_field, complex)
    for i, p in enumerate(P.ports):
        if i == q:
            Bm, bp = oracle.assemble_robin_bc_excited(fld, Bm, p.tri_ids, lambda x, y, z, p=p: p.get_Uinc(x, y, z, k0),
                                                      p.get_gamma(k0), oracle.dunavant4())
            b += bp
        else:
            Bm = oracle.assemble_robin_bc(fld, Bm, p.tri_ids, p.get_gamma(k0))
    K = (E - B * k0 ** 2 + fld.generate_csr(Bm)).tocsc()
    ids = P.solve_ids
    x = np.zeros(fld.n_field, complex)
    x[ids] = spl.spsolve(K[ids][:, ids], b[ids])
    return x, K


def test_device_lu_solve_matches_superlu(cuda):
    P = problems.waveguide()
    sw = FrequencySweep(P)
    lu = DeviceLU(sw).factor(10e9)
    assert lu.n_perturbed == 0
    _, K, olu = _oracle_solutions(P, 10e9, [])
    ids = P.solve_ids
    rng = np.random.default_rng(3)
    b = np.zeros((sw.n, 3), complex)
    b[ids] = rng.standard_normal((len(ids), 3)) + 1j * rng.standard_normal((len(ids), 3))
    x = lu.solve(torch.from_numpy(b).to(sw.device)).cpu().numpy()
    for j in range(3):
        xr = olu.solve(b[ids, j])
        # complex64 factors: the error is the single-precision rounding amplified by the conditioning
        assert np.linalg.norm(x[ids, j] - xr) <= 1e-3 * np.linalg.norm(xr)
    pec = np.setdiff1d(np.arange(sw.n), ids)
    assert np.abs(x[pec]).max() == 0


def test_lu_preconditioned_sweep_matches_superlu_golden(cuda, golden):
    g = golden("config1")
    f = float(g["f"])
    P = problems.waveguide()
    sw = FrequencySweep(P)
    lu = DeviceLU(sw).factor(f)
    res = sw.solve_lu([(f, 0), (f, 1)], lu, tol=1e-12, maxit=60)
    assert (res.status == 0).all(), (res.status, res.iters, res.relres)
    assert res.iters.max() <= 12, res.iters            # the complex64 LU of the same operator: a few refinements
    x = res.x.cpu().numpy()
    for j, key in enumerate(("x1", "x2")):
        assert np.linalg.norm(x[:, j] - g[key]) <= 1e-10 * np.linalg.norm(g[key])
    # the same factorization preconditions a neighbouring frequency
    f2 = 1.03 * f
    r2 = sw.solve_lu([(f2, 0), (f2, 1)], lu, tol=1e-10, maxit=300)
    assert (r2.status == 0).all(), (r2.status, r2.iters, r2.relres)
    xs, _, _ = _oracle_solutions(P, f2, [0, 1])
    for q in (0, 1):
        assert np.linalg.norm(r2.x[:, q].cpu().numpy() - xs[q]) <= 1e-8 * np.linalg.norm(xs[q])


def test_lu_solves_a_cavity_where_block_jacobi_stalls(cuda):
    """The dielectric-loaded cavity family (closed, lightly lossy, one port): block-Jacobi BiCGStab does
    not reach 1e-8, the LU-preconditioned solve does and agrees with SuperLU."""
    P = problems.cavity(n=8)
    sw = FrequencySweep(P)
    freqs = [float(f) for f in P.freqs[40:44]]
    systems = [(f, 0) for f in freqs]
    bj = sw.solve(systems, tol=1e-8, maxit=4000, precond="block_jacobi")
    lu = DeviceLU(sw).factor(freqs[1])
    res = sw.solve_lu(systems, lu, tol=1e-10, maxit=400)
    assert (res.status == 0).all(), (res.status, res.iters, res.relres)
    assert (bj.status != 0).any() or bj.iters.max() > 20 * res.iters.max()
    for j, f in enumerate(freqs):
        xr, _ = _oracle_solution(P, f, 0)
        assert np.linalg.norm(res.x[:, j].cpu().numpy() - xr) <= 1e-8 * np.linalg.norm(xr), f


def test_partitioned_entry_points_on_one_rank(cuda):
    """FrequencySweep.solve_partitioned (windows of the direct sweep, or Krylov batches) and the multi-mesh
    solve_meshes_partitioned give, on a single rank, what the unpartitioned calls give."""
    from emerge_b200.batch import solve_meshes_partitioned
    P = problems.waveguide(nx=6, ny=3, nz=10)
    sw = FrequencySweep(P)
    systems = [(f, q) for f in (9e9, 9.5e9, 10e9, 10.5e9) for q in (0, 1)]
    got = sw.solve_partitioned(systems, solver="direct", window=2, tol=1e-10)
    ref = sw.solve_direct(systems, window=2, tol=1e-10)
    assert [d["status"] for d in got] == [0] * len(systems)
    assert [d["iters"] for d in got] == ref.iters.tolist()
    got_k = sw.solve_partitioned(systems[:4], solver="krylov", tol=1e-8, precond="aux", return_x=True)
    assert all(d["status"] == 0 and d["relres"] <= 1e-8 for d in got_k)
    Ps = [problems.waveguide(nx=n, ny=3, nz=2 * n, seed=n) for n in (4, 6, 5)]
    sl = [[(10e9, 0), (10e9, 1)] for _ in Ps]
    out = solve_meshes_partitioned(Ps, sl, tol=1e-8, maxit=20000, precond="aux")
    assert len(out) == 3 and all(d["status"] == 0 for per in out for d in per)


def _substrate_direct(P, f):
    """SuperLU on the oracle's K_f of a substrate box (lumped ports, order-2 ABC) for port 1."""
    from oracle import abc2 as oabc2
    k0 = k0_of(f)
    E, B = oracle.tet_mass_stiffness_matrices(P.field, P.er, P.ur)
    Bm = P.field.empty_tri_matrix()
    pvs = []
    for p in P.ports:
        Bm, bp = oracle.assemble_robin_bc_excited(P.field, Bm, p.tri_ids, lambda x, y, z, p=p: p.get_Uinc(x, y, z, k0),
                                                  p.get_gamma(k0), oracle.dunavant4())
        pvs.append(bp)
    for bc in P.robin:
        Bm = oracle.assemble_robin_bc(P.field, Bm, bc.tri_ids, bc.get_gamma(k0))
        Bm = Bm + oabc2.abc_order_2_matrix(P.field, bc.tri_ids, bc.get_gamma2(k0))
    K = (E - B * k0 ** 2 + P.field.generate_csr(Bm)).tocsr()
    return oracle.solve_routine(K, pvs[:1], P.solve_ids)[0]


def test_complex128_factorization_at_low_frequency_matches_superlu(cuda):
    """The complex128 factorization (emfem_mf_set_precision 128, complex64 factor store) of an
    equilibrated substrate box at 1 GHz, where the gradient near-null space is strongest, under FP64
    BiCGStab: the oracle's SuperLU solution to 1e-10, within a few iterations."""
    P = problems.substrate_box(10, 8, 10)
    sw = FrequencySweep(P)
    lu = sw.direct_solver()
    bytes64 = lu.device_bytes
    lu.set_precision("c128")
    assert lu.device_bytes > bytes64
    f = 1e9
    lu.factor(f)
    r = sw.solve_lu([(f, 0)], lu, tol=1e-12, maxit=40)
    assert r.status[0] == 0 and r.iters[0] <= 10, (r.status, r.iters, r.relres)
    xs = _substrate_direct(P, f)
    x = r.x[:, 0].cpu().numpy()
    assert np.linalg.norm(x - xs) <= 1e-10 * np.linalg.norm(xs)
    lu.set_precision("c64")
    assert lu.device_bytes == bytes64 and lu.frequency is None


def test_auto_precision_sweep_converges_every_frequency(cuda):
    """solve_direct(precision="auto") over 1-8 GHz of a substrate box: every system converges to the
    FP64 tolerance, and the solutions at the lowest and highest frequency match the oracle's SuperLU."""
    P = problems.substrate_box(10, 8, 10)
    sw = FrequencySweep(P)
    freqs = [1e9, 1.5e9, 2e9, 4e9, 6e9, 8e9]
    systems = [(f, 0) for f in freqs]
    r = sw.solve_direct(systems, window=3, tol=1e-10, precision="auto")
    assert (r.status == 0).all() and (r.relres <= 1e-10).all(), (r.status, r.iters, r.relres, r.windows)
    assert {w["precision"] for w in r.windows} <= {"c64", "c128"}
    for j in (0, len(freqs) - 1):
        xs = _substrate_direct(P, freqs[j])
        x = r.x[:, j].cpu().numpy()
        assert np.linalg.norm(x - xs) <= 1e-8 * np.linalg.norm(xs), freqs[j]
