"""The CPU oracle against golden vectors produced by the reference's own numba code
(tests/golden/make_golden.py).  This pins the oracle that the GPU parity tests rely on."""
import hashlib

import numpy as np
import pytest

import oracle
from conftest import rel_fro_per_row
from emerge_b200 import problems
from emerge_b200.mesh import TetMesh
from emerge_b200.nedelec2 import Nedelec2
from emerge_b200.ports import PortFrame, RectangularWaveguidePort, k0_of


@pytest.fixture(scope="module")
def small(golden):
    d = golden("element_small")
    m = TetMesh(d["nodes"], d["tets"])
    return d, m, Nedelec2(m)


def test_element_matrices_match_reference(small):
    d, m, f = small
    dE, dB, r, c = oracle.matrix_builder(m.nodes, m.tets, m.tris, m.edges, m.edge_lengths, f.tet_to_field,
                                         m.tet_to_edge, d["ur"], d["er"])
    nt = m.n_tets
    assert rel_fro_per_row(dE.reshape(nt, 400), d["dataE"].reshape(nt, 400)) <= 1e-13
    assert rel_fro_per_row(dB.reshape(nt, 400), d["dataB"].reshape(nt, 400)) <= 1e-13
    assert np.array_equal(r, d["rows"]) and np.array_equal(c, d["cols"])


def test_csr_matches_reference(small):
    d, m, f = small
    E, B = oracle.tet_mass_stiffness_matrices(f, d["er"], d["ur"])
    assert np.array_equal(E.indptr, d["E_indptr"]) and np.array_equal(E.indices, d["E_indices"])
    assert np.array_equal(B.indptr, d["B_indptr"]) and np.array_equal(B.indices, d["B_indices"])
    assert np.abs(E.data - d["E_data"]).max() <= 1e-12 * np.abs(d["E_data"]).max()
    assert np.abs(B.data - d["B_data"]).max() <= 1e-12 * np.abs(d["B_data"]).max()


def test_robin_matches_reference(small, golden):
    d, m, f = small
    rb = golden("robin_small")
    a, b, l = 1.0e-2, 0.8e-2, 1.3e-2
    k0 = float(rb["k0"])
    p1 = RectangularWaveguidePort(1, PortFrame((a / 2, b / 2, 0.0)), (a, b), rb["tris_port1"])
    assert p1.get_beta(k0) == pytest.approx(float(rb["beta"]), rel=1e-15)
    assert p1.Zmode(k0) == pytest.approx(float(rb["Zmode"]), rel=1e-15)
    assert np.array_equal(oracle.dunavant4(), rb["DPTs"])
    Bm = f.empty_tri_matrix()
    Bm, bv = oracle.assemble_robin_bc_excited(f, Bm, rb["tris_port1"], lambda x, y, z: p1.get_Uinc(x, y, z, k0),
                                              p1.get_gamma(k0), oracle.dunavant4())
    Bm = oracle.assemble_robin_bc(f, Bm, rb["tris_port2"], complex(rb["gamma2"]))
    blk = Bm.reshape(-1, 64)[rb["touched"]]
    assert np.abs(blk - rb["blocks"]).max() <= 1e-14 * np.abs(rb["blocks"]).max()
    assert np.abs(bv - rb["bvec"]).max() <= 1e-14 * np.abs(rb["bvec"]).max()


def test_config1_pattern_and_solution_match_reference(golden):
    g = golden("config1")
    P = problems.waveguide()
    assert hashlib.sha256(P.mesh.nodes.tobytes()).hexdigest() == str(g["nodes_sha"])
    E, B = oracle.tet_mass_stiffness_matrices(P.field, P.er, P.ur)
    assert E.nnz == int(g["E_nnz"]) and np.array_equal(E.indptr, g["E_indptr"])
    assert hashlib.sha256(E.indices.astype(np.int32).tobytes()).hexdigest() == str(g["E_indices_sha"])
    s = g["samp"]
    assert np.abs(E.data[s] - g["E_samp"]).max() <= 1e-12 * np.abs(g["E_samp"]).max()
    assert np.abs(B.data[s] - g["B_samp"]).max() <= 1e-12 * np.abs(g["B_samp"]).max()
    k0 = k0_of(float(g["f"]))
    K = (E - B * k0 ** 2).tocsr()
    Bm = P.field.empty_tri_matrix()
    pvs = []
    for p in P.ports:
        Bm, bp = oracle.assemble_robin_bc_excited(P.field, Bm, p.tri_ids, lambda x, y, z, p=p: p.get_Uinc(x, y, z, k0),
                                                  p.get_gamma(k0), oracle.dunavant4())
        pvs.append(bp)
    K = K + P.field.generate_csr(Bm)
    assert K.nnz == int(g["K_nnz"])
    for pv, key in zip(pvs, ("pv1", "pv2")):
        idx = np.flatnonzero(pv)
        assert np.array_equal(idx, g[key + "_idx"])
        assert np.abs(pv[idx] - g[key + "_val"]).max() <= 1e-13 * np.abs(g[key + "_val"]).max()
    sid = P.solve_ids
    assert len(sid) == int(g["n_solve"])
    xs = oracle.solve_routine(K, pvs, sid)
    for x, gx in zip(xs, (g["x1"], g["x2"])):
        assert np.linalg.norm(x - gx) / np.linalg.norm(gx) <= 1e-10


def test_sparam_oracle_matches_reference(golden):
    """The S-parameter oracle, fed the reference's own SuperLU solutions, reproduces the reference's
    raw S-matrix (sparam_field_power / sparam_mode_power with ned2_tet_interp)."""
    from oracle import sparams as osp
    g = golden("config1")
    P = problems.waveguide()
    S = osp.sparams(P, {0: g["x1"], 1: g["x2"]}, k0_of(float(g["f"])), oracle.dunavant4())
    assert np.abs(S - g["S"]).max() <= 1e-12


CONN_KEYS = ("edges", "tris", "tet_to_edge", "tet_to_tri", "tri_to_edge", "tri_to_tet")


@pytest.mark.parametrize("case", ["a", "b"])
def test_connectivity_oracle_and_host_mesh_match_reference(golden, case):
    """oracle.connectivity and the host TetMesh reproduce Mesh3D._pre_update's arrays exactly."""
    from oracle import connectivity as oc
    g = golden("mesh_conn")
    nodes, tets = g[case + "_nodes"], g[case + "_tets"]
    o = oc.connectivity(nodes, tets)
    m = TetMesh(nodes, tets)
    for k in CONN_KEYS:
        assert np.array_equal(o[k], g[case + "_" + k]), k
        assert np.array_equal(getattr(m, k), g[case + "_" + k]), k
    assert np.array_equal(o["edge_lengths"], g[case + "_edge_lengths"])
    assert np.abs(m.edge_lengths - g[case + "_edge_lengths"]).max() <= 1e-15
