"""GPU parity of the Robin/port kernel, the frequency assembly and the batched COCG solve."""
import numpy as np
import pytest
import torch

import oracle
from emerge_b200 import assembly, problems
from emerge_b200.assembler import Assembler
from emerge_b200.mesh import TetMesh
from emerge_b200.nedelec2 import Nedelec2
from emerge_b200.ports import PortFrame, RectangularWaveguidePort, k0_of
from emerge_b200.solver import SolveRoutine, SolverB200COCG, SolverB200Krylov
from emerge_b200.sweep import FrequencySweep

pytestmark = pytest.mark.gpu


def test_robin_kernel_vs_reference_golden(cuda, golden):
    d = golden("element_small")
    rb = golden("robin_small")
    m = TetMesh(d["nodes"], d["tets"])
    f = Nedelec2(m)
    a, b = 1.0e-2, 0.8e-2
    k0 = float(rb["k0"])
    p1 = RectangularWaveguidePort(1, PortFrame((a / 2, b / 2, 0.0)), (a, b), rb["tris_port1"])
    Bm = f.empty_tri_matrix()
    Bm, bv = assembly.assemble_robin_bc_excited(f, Bm, rb["tris_port1"], lambda x, y, z: p1.get_Uinc(x, y, z, k0),
                                                p1.get_gamma(k0), rb["DPTs"])
    Bm = assembly.assemble_robin_bc(f, Bm, rb["tris_port2"], complex(rb["gamma2"]))
    blk = Bm.reshape(-1, 64)[rb["touched"]]
    assert np.abs(blk - rb["blocks"]).max() <= 1e-12 * np.abs(rb["blocks"]).max()
    assert np.abs(bv - rb["bvec"]).max() <= 1e-12 * np.abs(rb["bvec"]).max()


def test_freq_assembly_vs_reference_golden(cuda, golden):
    g = golden("config1")
    P = problems.waveguide()
    job = Assembler().assemble_freq_matrix(P.field, P.er, P.ur, P.ports, P.pec_tris, float(g["f"]))
    assert job.A.nnz == int(g["K_nnz"])
    assert np.array_equal(job.A.indptr, g["K_indptr"])
    s = g["samp"]
    assert np.abs(job.A.data[s] - g["K_samp"]).max() <= 1e-12 * np.abs(g["K_samp"]).max()
    for key, pn in (("pv1", 1), ("pv2", 2)):
        pv = job.port_vectors[pn]
        idx = np.flatnonzero(pv)
        assert np.array_equal(idx, g[key + "_idx"])
        assert np.abs(pv[idx] - g[key + "_val"]).max() <= 1e-12 * np.abs(g[key + "_val"]).max()
    assert len(job.solve_ids) == int(g["n_solve"])


def test_device_combine_matches_scipy_arithmetic(cuda):
    """emfem_sweep_combine + the zero-dropping compaction against SciPy's E - B*K0**2 (+ generate_csr(Bempty))
    on the same device-assembled E and B (ASM/assembler.py:255, :350): the same CSR layout, and without
    boundary terms the same bits."""
    from emerge_b200.assembler import freq_matrix_device
    P = problems.waveguide()
    sw = FrequencySweep(P)
    k0 = k0_of(10e9)
    Eh, Bh = sw.plan.to_scipy(sw.E), sw.plan.to_scipy(sw.B)
    Kref = (Eh - Bh * (k0 ** 2)).tocsr()
    K = freq_matrix_device(sw.plan, sw.E, sw.B, k0 ** 2)
    assert np.array_equal(K.indptr, Kref.indptr) and np.array_equal(K.indices, Kref.indices)
    assert np.array_equal(K.data, Kref.data)
    # with the ports' Robin blocks: the drop-in Assembler against the same steps in SciPy
    job = Assembler().assemble_freq_matrix(P.field, P.er, P.ur, P.ports, P.pec_tris, 10e9)
    Bm = P.field.empty_tri_matrix()
    dpts = assembly.dunavant4()
    for p in P.ports:
        Bm, _ = assembly.assemble_robin_bc_excited(P.field, Bm, p.tri_ids,
                                                   lambda x, y, z, p=p: p.get_Uinc(x, y, z, k0), p.get_gamma(k0), dpts)
    Kp = (Kref + P.field.generate_csr(Bm)).tocsr()
    assert np.array_equal(job.A.indptr, Kp.indptr) and np.array_equal(job.A.indices, Kp.indices)
    assert np.abs(job.A.data - Kp.data).max() <= 1e-15 * np.abs(Kp.data).max()


def test_sweep_solve_matches_superlu_golden(cuda, golden):
    """Device COCG (FP64, block Jacobi) on the 6 000-tet guide vs the reference's SuperLU solution."""
    g = golden("config1")
    P = problems.waveguide()
    sw = FrequencySweep(P)
    f = float(g["f"])
    res = sw.solve([(f, 0), (f, 1)], tol=1e-12, maxit=60000, precond="block_jacobi")
    x = res.x.cpu().numpy()
    assert (res.status == 0).all(), (res.status, res.iters, res.relres)
    for j, key in enumerate(("x1", "x2")):
        gx = g[key]
        assert np.linalg.norm(x[:, j] - gx) / np.linalg.norm(gx) <= 1e-10


def test_mixed_precision_reaches_fp64_residual(cuda, golden):
    g = golden("config1")
    P = problems.waveguide()
    sw = FrequencySweep(P)
    f = float(g["f"])
    res = sw.solve([(f, 0), (f, 1)], tol=1e-8, maxit=60000, precision="mixed")
    assert (res.status == 0).all(), (res.status, res.iters, res.relres)
    assert (res.relres <= 1e-8).all()
    x = res.x.cpu().numpy()
    for j, key in enumerate(("x1", "x2")):
        gx = g[key]
        assert np.linalg.norm(x[:, j] - gx) / np.linalg.norm(gx) <= 1e-5


def test_solver_plugin_through_solve_routine(cuda, golden):
    g = golden("config1")
    P = problems.waveguide()
    job = Assembler().assemble_freq_matrix(P.field, P.er, P.ur, P.ports, P.pec_tris, float(g["f"]))
    assert SolverB200COCG is SolverB200Krylov
    routine = SolveRoutine(SolverB200Krylov(tol=1e-12, maxit=60000))
    for (A, b, ids, reuse, aux), key in zip(job.iter_Ab(), ("x1", "x2")):
        x, rep = routine.solve(A, b, ids, reuse=reuse)
        assert rep.exit_code == 0, rep.aux
        gx = g[key]
        assert np.linalg.norm(x - gx) / np.linalg.norm(gx) <= 1e-10


def test_abc2_kernel_vs_reference_golden(cuda, golden):
    g = golden("abc2")
    d = golden("element_small")
    f = Nedelec2(TetMesh(d["nodes"], d["tets"]))
    M = assembly.abc_order_2_matrix(f, g["tri_ids"], complex(g["cf"])).reshape(-1, 64)[g["tri_ids"]]
    assert np.abs(M - g["blocks"]).max() <= 1e-12 * np.abs(g["blocks"]).max()


@pytest.mark.parametrize("kind", ["abc", "abc2", "surface", "lumped"])
def test_sweep_with_robin_boundaries_matches_superlu(cuda, kind):
    """Non-excited Robin boundaries in the device sweep (an absorbing boundary in place of the
    second port; a conducting surface-impedance wall in place of a PEC wall) vs the oracle's
    assembly with assemble_robin_bc and SuperLU."""
    from emerge_b200.boundaries import AbsorbingBoundary, SurfaceImpedance
    P = problems.waveguide()
    m = P.mesh
    a, b, l = P.dims
    if kind == "lumped":
        from emerge_b200.ports import LumpedPort
        P.ports = [P.ports[0], LumpedPort(2, P.ports[1].tri_ids, width=a, height=b, direction=(0.0, 1.0, 0.0))]
    elif kind in ("abc", "abc2"):
        P.robin = [AbsorbingBoundary(P.ports[1].tri_ids, order=1 if kind == "abc" else 2)]
        P.ports = P.ports[:1]
    else:
        wall = m.tris_on_plane(1, b)
        P.pec_tris = np.setdiff1d(P.pec_tris, wall)
        P.robin = [SurfaceImpedance(wall, sigma=1.0e5, roughness=1e-6)]
    sw = FrequencySweep(P)
    f = 10e9
    sysl = [(f, q) for q in range(len(P.ports))]
    res = sw.solve(sysl, tol=1e-12, maxit=60000, precond="aux")
    assert (res.status == 0).all(), (res.status, res.iters, res.relres)
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
        if getattr(bc, "order", 1) == 2:
            from oracle import abc2 as oabc2
            Bm = Bm + oabc2.abc_order_2_matrix(P.field, bc.tri_ids, bc.get_gamma2(k0))
    K = K + P.field.generate_csr(Bm)
    xs = oracle.solve_routine(K, pvs, P.solve_ids)
    x = res.x.cpu().numpy()
    for j in range(len(P.ports)):
        assert np.linalg.norm(x[:, j] - xs[j]) / np.linalg.norm(xs[j]) <= 1e-10
    # the drop-in assembler with the same boundaries gives the same K
    job = Assembler().assemble_freq_matrix(P.field, P.er, P.ur, P.ports, P.pec_tris, f, robin_bcs=P.robin)
    d = (job.A - K).tocsr()
    assert (abs(d).max() if d.nnz else 0.0) <= 1e-12 * abs(K).max()
