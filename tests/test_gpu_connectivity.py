"""GPU mesh connectivity (emfem_mesh_connect_*) against Mesh3D._pre_update's own output and the
host TetMesh, plus the device checks for bad meshes."""
import numpy as np
import pytest
import torch

from emerge_b200 import assembly
from emerge_b200._lib import EmfemError
from emerge_b200.connectivity import DeviceTetMesh
from emerge_b200.mesh import TetMesh, box_tet_mesh
from emerge_b200.nedelec2 import Nedelec2

pytestmark = pytest.mark.gpu

KEYS = ("edges", "tris", "tet_to_edge", "tet_to_tri", "tri_to_edge", "tri_to_tet")


@pytest.mark.parametrize("case", ["a", "b"])
def test_device_connectivity_vs_reference_golden(cuda, golden, case):
    g = golden("mesh_conn")
    d = DeviceTetMesh(g[case + "_nodes"], g[case + "_tets"]).to_host()
    for k in KEYS:
        assert np.array_equal(d[k], g[case + "_" + k]), k
    assert np.array_equal(d["edge_lengths"], g[case + "_edge_lengths"])


def _permuted_box(n, seed):
    nodes, tets = box_tet_mesh(n, n - 3, n + 2, 0.03, 0.02, 0.04, jitter=0.12, seed=seed, shuffle_local=True)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(nodes.shape[1])
    nodes_p = np.empty_like(nodes)
    nodes_p[:, perm] = nodes
    return nodes_p, perm[tets][:, rng.permutation(tets.shape[1])]


@pytest.mark.parametrize("n,seed", [(9, 1), (40, 2)])
def test_device_connectivity_vs_host_mesh(cuda, n, seed):
    nodes, tets = _permuted_box(n, seed)
    m = TetMesh(nodes, tets)
    d = DeviceTetMesh(nodes, tets).to_host()
    for k in KEYS:
        assert np.array_equal(d[k], getattr(m, k)), k
    assert np.array_equal(d["edge_lengths"], m.edge_lengths)


def test_assembly_from_device_connectivity(cuda):
    """A mesh whose connectivity never left the GPU assembles to the same CSR as the host mesh."""
    nodes, tets = _permuted_box(8, 5)
    m = TetMesh(nodes, tets)
    nt = m.n_tets
    rng = np.random.default_rng(3)
    er = np.zeros((3, 3, nt), complex)
    ur = np.zeros((3, 3, nt), complex)
    for i in range(3):
        er[i, i] = rng.uniform(1, 4, nt) - 0.1j
        ur[i, i] = 1.0
    dm_host = assembly.DeviceMesh(m)
    dm_dev = assembly.DeviceMesh(DeviceTetMesh(nodes, tets))
    out = []
    for dm in (dm_host, dm_dev):
        plan = assembly.CsrPlan(dm)
        E, B = plan.assemble(er, ur)
        out.append((plan.host_pattern(), E.cpu().numpy(), B.cpu().numpy()))
    (p0, E0, B0), (p1, E1, B1) = out
    assert all(np.array_equal(a, b) for a, b in zip(p0, p1))
    assert np.array_equal(E0, E1) and np.array_equal(B0, B1)


def test_rejects_out_of_range_and_repeated_nodes(cuda):
    nodes, tets = box_tet_mesh(2, 2, 2, 1.0, 1.0, 1.0)
    bad = tets.copy()
    bad[2, 5] = nodes.shape[1]
    with pytest.raises(EmfemError):
        DeviceTetMesh(nodes, bad)
    rep = tets.copy()
    rep[1, 3] = rep[0, 3]
    with pytest.raises(EmfemError):
        DeviceTetMesh(nodes, rep)
    DeviceTetMesh(nodes, tets)          # the handle stays usable


def test_flags_triangle_shared_by_three_tets(cuda):
    nodes = np.array([[0, 1, 0, 0.3, 0.2, -0.4], [0, 0, 1, 0.3, -0.5, 0.2], [0, 0, 0, 1, -1, 0.7]], dtype=float)
    tets = np.array([[0, 1, 2, 3], [0, 1, 2, 4], [0, 1, 2, 5]]).T.copy()
    with pytest.raises(EmfemError, match="capacity"):
        DeviceTetMesh(nodes, tets)
