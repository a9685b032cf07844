"""Edge cases of the device path: the smallest meshes, the largest batches, degenerate requests."""
import numpy as np
import pytest
import torch

import oracle
from emerge_b200 import assembly, problems
from emerge_b200.auxspace import AuxSpace, Network
from emerge_b200.batch import MeshBatch
from emerge_b200.connectivity import DeviceTetMesh
from emerge_b200.mesh import TetMesh, box_tet_mesh
from emerge_b200.nedelec2 import Nedelec2
from emerge_b200.sweep import FrequencySweep

pytestmark = pytest.mark.gpu

ONE_TET = (np.array([[0.0, 1.0, 0.1, 0.2], [0.0, 0.1, 1.2, 0.3], [0.0, 0.2, 0.1, 0.9]]) * 1e-2,
           np.array([[2], [0], [3], [1]]))


def test_single_tet_assembly_connectivity_and_aux(cuda):
    nodes, tets = ONE_TET
    m = TetMesh(nodes, tets)
    f = Nedelec2(m)
    er = np.zeros((3, 3, 1), complex); ur = np.zeros((3, 3, 1), complex)
    for i in range(3):
        er[i, i] = 2.0 - 0.1j
        ur[i, i] = 1.0
    E, B = assembly.tet_mass_stiffness_matrices(f, er, ur)
    Eo, Bo = oracle.tet_mass_stiffness_matrices(f, er, ur)
    assert E.shape == (20, 20) and np.array_equal(E.indptr, Eo.indptr) and np.array_equal(E.indices, Eo.indices)
    assert np.abs(E.data - Eo.data).max() <= 1e-12 * np.abs(Eo.data).max()
    assert np.abs(B.data - Bo.data).max() <= 1e-12 * np.abs(Bo.data).max()
    d = DeviceTetMesh(nodes, tets).to_host()
    for k in ("edges", "tris", "tet_to_edge", "tet_to_tri", "tri_to_edge", "tri_to_tet"):
        assert np.array_equal(d[k], getattr(m, k)), k
    aux = AuxSpace(m)
    assert aux.n_aux == 4 + 6
    net = Network(aux, seed=0, init="random")
    x = torch.randn(aux.n_aux, 1, dtype=torch.complex64, device="cuda")
    assert torch.isfinite(torch.view_as_real(net.forward(x))).all()
    assert torch.isfinite(torch.view_as_real(net.infer(x))).all()


def test_batch_of_one_mesh_equals_single_assembly(cuda):
    nodes, tets = box_tet_mesh(2, 3, 2, 1e-2, 1e-2, 1e-2, jitter=0.1, seed=5)
    nt = tets.shape[1]
    rng = np.random.default_rng(1)
    er = np.zeros((3, 3, nt), complex); ur = np.zeros((3, 3, nt), complex)
    for i in range(3):
        er[i, i] = rng.uniform(1, 5, nt)
        ur[i, i] = 1.0
    b = MeshBatch([(nodes, tets)])
    b.assemble(torch.from_numpy(er).cuda(), torch.from_numpy(ur).cuda())
    E, _ = assembly.tet_mass_stiffness_matrices(Nedelec2(TetMesh(nodes, tets)), er, ur)
    Y = b.csr(0, "E")
    assert np.array_equal(Y.indptr, E.indptr) and np.array_equal(Y.indices, E.indices) and np.array_equal(Y.data, E.data)


def test_largest_batch_of_systems(cuda):
    """64 systems (the per-launch maximum) in one batched solve, the last ones duplicates of the
    first: identical systems give identical results (independent per-system scalars)."""
    P = problems.waveguide(nx=4, ny=2, nz=8, seed=1)
    sw = FrequencySweep(P)
    freqs = np.linspace(8.5e9, 11.5e9, 16)
    sysl = [(float(f), q) for f in freqs for q in (0, 1)]
    sysl = sysl + sysl
    res = sw.solve(sysl, tol=1e-10, maxit=20000, precond="aux")
    assert len(sysl) == 64 and (res.status == 0).all()
    x = res.x.cpu().numpy()
    assert np.array_equal(x[:, :32], x[:, 32:])
    with pytest.raises(AssertionError):
        sw.solve(sysl + sysl[:1], tol=1e-8)
