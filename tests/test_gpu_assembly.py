"""GPU parity of the tet integrator, the device CSR plan and the fused assembly (through the C ABI)."""
import ctypes
import hashlib

import numpy as np
import pytest
import torch

import oracle
from conftest import rel_fro_per_row
from emerge_b200 import assembly, problems
from emerge_b200.mesh import TetMesh, box_tet_mesh
from emerge_b200.nedelec2 import Nedelec2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(golden):
    d = golden("element_small")
    m = TetMesh(d["nodes"], d["tets"])
    return d, m, Nedelec2(m)


def test_element_kernel_vs_reference_golden(cuda, small):
    d, m, f = small
    dE, dB, r, c = assembly._matrix_builder(m.nodes, m.tets, m.tris, m.edges, m.edge_lengths, f.tet_to_field,
                                            m.tet_to_edge, d["ur"], d["er"])
    nt = m.n_tets
    assert rel_fro_per_row(dE.reshape(nt, 400), d["dataE"].reshape(nt, 400)) <= 1e-12
    assert rel_fro_per_row(dB.reshape(nt, 400), d["dataB"].reshape(nt, 400)) <= 1e-12
    assert np.array_equal(r, d["rows"]) and np.array_equal(c, d["cols"])


def test_plan_csr_vs_reference_golden(cuda, small):
    d, m, f = small
    E, B = assembly.tet_mass_stiffness_matrices(f, d["er"], d["ur"])
    assert np.array_equal(E.indptr, d["E_indptr"]) and np.array_equal(E.indices, d["E_indices"])
    assert np.array_equal(B.indptr, d["B_indptr"]) and np.array_equal(B.indices, d["B_indices"])
    assert np.abs(E.data - d["E_data"]).max() <= 1e-12 * np.abs(d["E_data"]).max()
    assert np.abs(B.data - d["B_data"]).max() <= 1e-12 * np.abs(d["B_data"]).max()


@pytest.mark.parametrize("shuffle", [False, True])
def test_plan_vs_oracle_random_tensors(cuda, shuffle):
    nodes, tets = box_tet_mesh(6, 5, 7, 0.02, 0.017, 0.03, jitter=0.12, seed=4, shuffle_local=shuffle)
    m = TetMesh(nodes, tets)
    f = Nedelec2(m)
    rng = np.random.default_rng(9)
    nt = m.n_tets
    er = rng.uniform(0.5, 2, (3, 3, nt)) + 1j * rng.uniform(-0.3, 0.3, (3, 3, nt))
    ur = rng.uniform(0.5, 2, (3, 3, nt)) + 1j * rng.uniform(-0.3, 0.3, (3, 3, nt))
    for i in range(3):
        er[i, i] += 3
        ur[i, i] += 3
    E, B = assembly.tet_mass_stiffness_matrices(f, er, ur)
    Eo, Bo = oracle.tet_mass_stiffness_matrices(f, er, ur)
    assert np.array_equal(E.indptr, Eo.indptr) and np.array_equal(E.indices, Eo.indices)
    for X, Xo in ((E, Eo), (B, Bo)):
        rows = np.repeat(np.arange(X.shape[0]), np.diff(X.indptr))
        rowmax = np.maximum.reduceat(np.abs(Xo.data), Xo.indptr[:-1])
        assert np.max(np.abs(X.data - Xo.data) / rowmax[rows]) <= 1e-12


def test_config1_assembly_vs_reference_golden(cuda, golden):
    g = golden("config1")
    P = problems.waveguide()
    E, B = assembly.tet_mass_stiffness_matrices(P.field, P.er, P.ur)
    assert E.nnz == int(g["E_nnz"]) and np.array_equal(E.indptr, g["E_indptr"])
    assert hashlib.sha256(E.indices.astype(np.int32).tobytes()).hexdigest() == str(g["E_indices_sha"])
    s = g["samp"]
    assert np.abs(E.data[s] - g["E_samp"]).max() <= 1e-12 * np.abs(g["E_samp"]).max()
    assert np.abs(B.data[s] - g["B_samp"]).max() <= 1e-12 * np.abs(g["B_samp"]).max()
    assert abs(np.linalg.norm(E.data) - float(g["E_fro"])) <= 1e-12 * float(g["E_fro"])


def test_fused_assembly_is_deterministic(cuda):
    P = problems.waveguide()
    dm = assembly.DeviceMesh(P.mesh, P.field)
    plan = assembly.CsrPlan(dm)
    E1, B1 = plan.assemble(P.er, P.ur)
    E2, B2 = plan.assemble(P.er, P.ur)
    assert torch.equal(E1, E2) and torch.equal(B1, B2)


def test_every_kernel_variant_gives_identical_values(cuda):
    """All assembly variants (chunk sizes, invariants staged in shared memory or read through L1)
    sum the same contributions in the same order: bit-identical E and B."""
    nodes, tets = box_tet_mesh(7, 6, 5, 0.02, 0.017, 0.03, jitter=0.12, seed=12, shuffle_local=True)
    m = TetMesh(nodes, tets)
    f = Nedelec2(m)
    rng = np.random.default_rng(4)
    nt = m.n_tets
    er = rng.uniform(0.5, 2, (3, 3, nt)) + 1j * rng.uniform(-0.3, 0.3, (3, 3, nt))
    ur = rng.uniform(0.5, 2, (3, 3, nt)) + 1j * rng.uniform(-0.3, 0.3, (3, 3, nt))
    for i in range(3):
        er[i, i] += 3
        ur[i, i] += 3
    dm = assembly.DeviceMesh(m, f)
    plan = assembly.CsrPlan(dm)
    n = ctypes.c_int()
    from emerge_b200._lib import lib as _l
    _l().emfem_plan_variants(plan._p, ctypes.byref(n), None)
    assert n.value >= 13
    ref = None
    for v in range(n.value):
        if not plan.variant_info(v)["available"]:
            continue
        plan.set_variant(v)
        E, B = plan.assemble(er, ur)
        cur = (E.cpu().numpy(), B.cpu().numpy())
        if ref is None:
            ref = cur
        else:
            assert np.array_equal(cur[0], ref[0]) and np.array_equal(cur[1], ref[1]), v


def test_drop_in_results_never_alias(cuda, small):
    """tet_mass_stiffness_matrices hands out pinned pool buffers: a result held by the caller keeps
    its values across later calls, and a released buffer is reused."""
    d, m, f = small
    E1, B1 = assembly.tet_mass_stiffness_matrices(f, d["er"], d["ur"])
    keep = E1.data.copy()
    view = B1.data[5:9]
    er2 = d["er"] * 2.0
    for _ in range(6):                       # more calls than pool buffers while E1/B1 are held
        E2, B2 = assembly.tet_mass_stiffness_matrices(f, er2, d["ur"])
    assert np.array_equal(E1.data, keep)
    np.testing.assert_array_equal(view, B1.data[5:9])
    assert not np.shares_memory(E1.data, E2.data) and not np.shares_memory(B1.data, B2.data)
    assert np.abs(B2.data - 2.0 * B1.data).max() <= 1e-12 * np.abs(B1.data).max()   # B is linear in er
