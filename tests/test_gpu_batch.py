"""Several uneven meshes assembled in one launch (MeshBatch): every mesh's E and B, sliced from the
union, equal a separate assembly of that mesh bit for bit."""
import numpy as np
import pytest
import torch

from emerge_b200 import assembly
from emerge_b200.batch import MeshBatch
from emerge_b200.mesh import TetMesh, box_tet_mesh
from emerge_b200.nedelec2 import Nedelec2

pytestmark = pytest.mark.gpu


def test_union_assembly_matches_separate_assembly(cuda):
    rng = np.random.default_rng(8)
    specs = [(3, 2, 4, 1.0e-2, 0.6e-2, 1.4e-2), (5, 3, 2, 2.0e-2, 1.0e-2, 0.7e-2), (2, 2, 2, 0.5e-2, 0.5e-2, 0.5e-2)]
    meshes, ers, urs = [], [], []
    for i, (nx, ny, nz, a, b, l) in enumerate(specs):
        nodes, tets = box_tet_mesh(nx, ny, nz, a, b, l, jitter=0.12, seed=30 + i, shuffle_local=True)
        meshes.append((nodes, tets))
        nt = tets.shape[1]
        er = np.zeros((3, 3, nt), complex)
        ur = np.zeros((3, 3, nt), complex)
        for d in range(3):
            er[d, d] = rng.uniform(1, 12, nt) * (1 - 1j * rng.uniform(0, 5e-3, nt))
            ur[d, d] = np.where(rng.random(nt) < 0.1, rng.uniform(1, 2, nt), 1.0)
        ers.append(er); urs.append(ur)
    batch = MeshBatch(meshes)
    er = torch.from_numpy(np.concatenate(ers, axis=2)).cuda()
    ur = torch.from_numpy(np.concatenate(urs, axis=2)).cuda()
    batch.assemble(er, ur)
    assert batch.n_tets == sum(t.shape[1] for _, t in meshes)
    for k, (nodes, tets) in enumerate(meshes):
        f = Nedelec2(TetMesh(nodes, tets))
        E, B = assembly.tet_mass_stiffness_matrices(f, ers[k], urs[k])
        for X, which in ((E, "E"), (B, "B")):
            Y = batch.csr(k, which)
            assert Y.shape == X.shape
            assert np.array_equal(Y.indptr, X.indptr) and np.array_equal(Y.indices, X.indices)
            assert np.array_equal(Y.data, X.data)
