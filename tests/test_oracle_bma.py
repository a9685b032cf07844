"""Port-mode (boundary-mode analysis) oracle and host logic against the reference's own outputs."""
import numpy as np
import scipy.sparse as sp

from oracle import bma as ob
from emerge_b200 import modal
from _bma_common import dof_permutation, guide_mesh, wall_edges


def test_element_blocks_match_reference(golden):
    g = golden("bma")
    A, B = ob.element_matrices(g["el_nodes"], g["el_tris"], g["el_edges"], g["el_t2f"][:3], g["el_er"],
                               g["el_ur"], float(g["el_k0"]))
    nt = A.shape[0]
    assert np.abs(A.reshape(nt, 196) - g["el_A"]).max() <= 1e-13 * np.abs(g["el_A"]).max()
    assert np.abs(B.reshape(nt, 196) - g["el_B"]).max() <= 1e-13 * np.abs(g["el_B"]).max()
    # the reference's quirks are present: zero A outside the transverse block, zero face-face Dtt
    assert np.all(g["el_A"].reshape(nt, 14, 14)[:, 8:, :] == 0)
    assert np.all(g["el_B"].reshape(nt, 14, 14)[:, [3, 7]][:, :, [3, 7]] == 0)
    _, _, rows, cols = ob.matrix_builder(g["el_nodes"], g["el_tris"], g["el_edges"], g["el_t2f"], g["el_ur"],
                                         g["el_er"], float(g["el_k0"]))
    assert np.array_equal(rows, g["el_rows"].ravel()) and np.array_equal(cols, g["el_cols"].ravel())


def test_port_surface_and_field_numbering(golden):
    g = golden("bma")
    s = modal.PortSurface(guide_mesh(g), g["wg_tri_ids"], modal.PortFrame())
    assert np.array_equal(s.tris, g["wg_sm_tris"]) and np.array_equal(s.nodes, g["wg_sm_nodes"])
    # same edges, lexicographic here: every reference triangle's edges map onto ours
    p = dof_permutation(g, s)
    ne = s.n_edges
    assert np.array_equal(p[:ne][g["wg_sm_tri_to_edge"]], s.tri_to_edge)
    f = modal.NedLeg2Field(s)
    assert f.n_field == int(g["wg_n_field"])
    assert np.array_equal(p[g["wg_tri_to_field"]], f.tri_to_field)
    # PEC DOFs of the walls: the same set as the reference's
    pec = np.ones(f.n_field, bool)
    pec[p[g["wg_solve_ids"]]] = False
    se = s.from_source_edges(wall_edges(guide_mesh(g), g))
    mine = np.zeros(f.n_field, bool)
    mine[f.edge_to_field[:, se[se >= 0]].ravel()] = True
    assert np.array_equal(pec, mine)


def test_eig_boundary_on_oracle_matrices_matches_reference(golden):
    """Host eigen step (dense LAPACK + the reference's filter) on the oracle's matrices."""
    g = golden("bma")
    k0 = float(g["wg_k0"])
    s = modal.PortSurface(guide_mesh(g), g["wg_tri_ids"], modal.PortFrame())
    f = modal.NedLeg2Field(s)
    p = dof_permutation(g, s)
    solve_ids = np.sort(p[g["wg_solve_ids"]])
    for tag in ("air", "half"):
        er = g[f"wg_{tag}_er"]
        ur = np.zeros_like(er)
        for i in range(3):
            ur[i, i] = 1.0
        E, B = ob.generalized_eigenvalue_matrix(s.local_nodes, s.tris, s.edges, f.tri_to_field, f.n_field, er,
                                                ur, k0)
        ref = sp.csr_matrix((g[f"wg_{tag}_E_data"], g[f"wg_{tag}_indices"], g[f"wg_{tag}_indptr"]))
        Ep = E[np.ix_(p, p)]
        assert abs(Ep - ref).max() <= 1e-13 * abs(ref).max()
        target = 0.7 * k0 * (1.0 if tag == "air" else float(np.mean(np.diagonal(er).ravel().real)))
        lam, _ = modal.eig_boundary(E, B, solve_ids, 6, True, target, -1.0)
        lref = g[f"wg_{tag}_lambda"]
        assert lam.shape == lref.shape
        assert np.abs(np.sort_complex(lam) - np.sort_complex(lref)).max() <= 1e-9 * np.abs(lref).max()


def test_modal_port_dispersion_and_impedance_formulas():
    """ModalPort's beta(k0), Z_mode and U_inc scale follow microwave_bc.py:716-730 and :218-230."""
    from emerge_b200.constants import C0, EPS0, MU0, Z0
    from emerge_b200.ports import ModalPort
    f0 = 10e9
    k0m = 2 * np.pi * f0 / C0
    for mt in ("TE", "TM"):
        p = ModalPort(1, np.arange(3))
        p.modes = [modal.PortMode(np.ones(4, complex), k0m, 150.0 + 0j, f0, mt)]
        p.modes[0].norm_factor = 2.5
        for f in (8e9, 12e9):
            k0 = 2 * np.pi * f / C0
            beta = np.sqrt(150.0 ** 2 + k0 ** 2 * (1 - (f0 / f) ** 2))
            assert abs(p.get_beta(k0) - beta) <= 1e-12 * beta
            zm = k0 * C0 / beta * MU0 if mt == "TE" else beta / (k0 * C0 * EPS0)
            assert abs(p.Zmode(k0) - zm) <= 1e-12 * zm
            assert abs(p.uinc_scale(k0) - (-2j * beta * np.sqrt(zm / Z0) * 2.5)) <= 1e-12 * abs(p.uinc_scale(k0))
    p = ModalPort(1, np.arange(3), TEM=True)
    p.modes = [modal.PortMode(np.ones(4, complex), k0m, 1.2 * k0m + 0j, f0, "TEM")]
    assert abs(p.get_beta(2 * k0m) - 2.4 * k0m) <= 1e-12 * k0m and p.Zmode(k0m) == Z0
