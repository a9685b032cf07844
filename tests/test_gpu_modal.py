"""Port-mode analysis on the device: triangle blocks, port-face CSR, eigenvalues and modes against
the reference's own outputs, and the TE10 mode of a rectangular guide against its closed form."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from emerge_b200 import modal
from emerge_b200._lib import EmfemError
from _bma_common import dof_permutation, guide_mesh, wall_edges

pytestmark = pytest.mark.gpu


class _Surf:
    """A PortSurface stand-in carrying the fixture's raw arrays (random orientations)."""

    def __init__(self, g):
        self.local_nodes = g["el_nodes"]
        self.tris = g["el_tris"]
        self.edges = g["el_edges"]
        self.tri_to_edge = g["el_t2f"][:3]
        self.n_nodes = self.local_nodes.shape[1]
        self.n_edges = self.edges.shape[1]
        self.n_tris = self.tris.shape[1]


def test_triangle_blocks_match_reference(cuda, golden):
    g = golden("bma")
    A, B = modal.bma_blocks(_Surf(g), g["el_er"], g["el_ur"], float(g["el_k0"]), cuda)
    A, B = A.cpu().numpy(), B.cpu().numpy()
    assert np.abs(A - g["el_A"]).max() <= 1e-12 * np.abs(g["el_A"]).max()
    assert np.abs(B - g["el_B"]).max() <= 1e-12 * np.abs(g["el_B"]).max()


@pytest.mark.parametrize("tag", ["air", "half"])
def test_port_face_matrices_eigenvalues_and_mode(cuda, golden, tag):
    g = golden("bma")
    m = guide_mesh(g)
    k0 = float(g["wg_k0"])
    er = g[f"wg_{tag}_er"]
    ur = np.zeros_like(er)
    for i in range(3):
        ur[i, i] = 1.0
    E, B, solve_ids, fld = modal.assemble_bma_matrices(m, g["wg_tri_ids"], modal.PortFrame(), er, ur, k0,
                                                       pec_edges=wall_edges(m, g), device=cuda)
    p = dof_permutation(g, fld.mesh)
    refE = sp.csr_matrix((g[f"wg_{tag}_E_data"], g[f"wg_{tag}_indices"], g[f"wg_{tag}_indptr"]))
    refB = sp.csr_matrix((g[f"wg_{tag}_B_data"], g[f"wg_{tag}_indices"], g[f"wg_{tag}_indptr"]))
    Ep, Bp = E[np.ix_(p, p)], B[np.ix_(p, p)]
    assert Ep.nnz == refE.nnz
    assert abs(Ep - refE).max() <= 1e-12 * abs(refE).max()
    assert abs(Bp - refB).max() <= 1e-12 * abs(refB).max()
    assert np.array_equal(np.sort(p[g["wg_solve_ids"]]), solve_ids)

    target = 0.7 * k0 * (1.0 if tag == "air" else float(np.mean(np.diagonal(er).ravel().real)))
    lam, vecs = modal.eig_boundary(E, B, solve_ids, 6, True, target, -1.0)
    lref = g[f"wg_{tag}_lambda"]
    assert np.abs(np.sort_complex(lam) - np.sort_complex(lref)).max() <= 1e-9 * np.abs(lref).max()

    modes, fld2 = modal.modal_analysis(m, g["wg_tri_ids"], modal.PortFrame(), er, ur, 10e9, pec_edges=wall_edges(m, g),
                                       target_kz=target, device=cuda)
    top = modes[0]
    assert abs(top.beta ** 2 + lref[np.argmax(np.sqrt(-lref).real)]) <= 1e-9 * np.abs(lref).max()
    # the reference's top eigenvector, phase-normalised like modal_analysis (MW/microwave_3d.py:581-584)
    ref = np.zeros(fld2.n_field, complex)
    ref[p[g["wg_solve_ids"]]] = g[f"wg_{tag}_mode"]
    ref = ref * np.exp(-1j * np.angle(ref[np.argmax(np.abs(ref))]))
    mine = top.modefield
    s = np.sign(np.real(np.vdot(ref, mine)))
    assert np.abs(s * mine - ref).max() <= 1e-8 * np.abs(ref).max()
    # the reference's type rule (MW/microwave_3d.py:640-646): the half-filled guide's dominant mode is
    # hybrid, with |E_z| above a tenth of |E_t|, so it is labelled TM
    ratio = np.abs(ref[fld2.n_xy:]).max() / np.abs(ref[:fld2.n_xy]).max()
    assert top.modetype == ("TE" if ratio < 0.1 else "TM")
    assert top.modetype == ("TE" if tag == "air" else "TM")
    if tag == "air":
        # TE10 of the 22.86 mm guide at 10 GHz: beta = sqrt(k0^2 - (pi/a)^2) within discretisation error
        exact = np.sqrt(k0 ** 2 - (np.pi / float(g["wg_a"])) ** 2)
        assert abs(top.beta.real - exact) / exact < 5e-3


def test_degenerate_triangle_is_reported(cuda, golden):
    g = golden("bma")
    s = _Surf(g)
    s.local_nodes = s.local_nodes.copy()
    t0 = s.tris[:, 0]
    s.local_nodes[:2, t0[2]] = s.local_nodes[:2, t0[0]]         # two coincident vertices: zero area
    with pytest.raises(EmfemError):
        modal.bma_blocks(s, g["el_er"], g["el_ur"], float(g["el_k0"]), cuda)
    from emerge_b200._lib import Handle
    assert Handle.get(cuda).device_status() == 0     # reported once, then cleared; the context is usable
    assert torch.ones(4, device=cuda).sum().item() == 4.0


def _ref_surface_mode(g, cuda, tag="air"):
    m = guide_mesh(g)
    s = modal.PortSurface(m, g["wg_tri_ids"], modal.PortFrame())
    fld = modal.NedLeg2Field(s)
    p = dof_permutation(g, s)
    em = np.zeros(fld.n_field, complex)
    em[p] = g[f"wg_{tag}_emode"]
    return m, s, fld, em


@pytest.mark.parametrize("tag", ["air", "half"])
def test_mode_field_interpolation_and_power_match_reference(cuda, golden, tag):
    """E and the curl form of H at the face's order-4 points (ned2_tri_interp_full / _curl) and the
    power flux (compute_avg_power_flux) of the reference's own mode vector."""
    from emerge_b200.assembly import dunavant4
    g = golden("bma")
    m, s, fld, em = _ref_surface_mode(g, cuda, tag)
    dp = dunavant4()
    pts = np.einsum("cvs,vp->cps", s.nodes[:, s.tris], dp[1:4])               # (3, 6, nt)
    loc = modal._local_points(s, pts)
    beta = complex(g[f"wg_{tag}_beta"])
    E = modal.tri_field(s, fld, em, loc, "E", device=cuda).cpu().numpy()
    H = modal.tri_field(s, fld, em, loc, "H", beta, np.ones((3, s.n_tris)), device=cuda).cpu().numpy()
    # the fixture flattened the same (3, 6, nt) point array
    Er = g[f"wg_{tag}_interpE"].reshape(3, 6, s.n_tris)
    Hr = g[f"wg_{tag}_interpH"].reshape(3, 6, s.n_tris)
    assert np.abs(E - Er).max() <= 1e-12 * np.abs(Er).max()
    assert np.abs(H - Hr).max() <= 1e-12 * np.abs(Hr).max()
    ur = np.zeros((3, 3, s.n_tris), complex)
    for i in range(3):
        ur[i, i] = 1.0
    P = modal.mode_power(s, fld, em, float(g["wg_k0"]), ur, beta, cuda)
    Pr = complex(g[f"wg_{tag}_power"]).real
    assert abs(P - Pr) <= 1e-10 * abs(Pr)
    assert np.allclose(modal.face_normal(s), g["wg_normal"])


def test_modal_ports_in_a_sweep_match_the_analytic_port(cuda):
    """A WR-90 section driven by ModalPorts whose TE10 comes from the face eigen-analysis gives the
    analytic-port S-parameters to within the 2-D mode's discretisation error."""
    from emerge_b200 import problems
    from emerge_b200.ports import ModalPort
    from emerge_b200.sweep import FrequencySweep
    P = problems.waveguide()
    f = 10e9
    ref = FrequencySweep(P)
    r0 = ref.solve([(f, 0), (f, 1)], tol=1e-10, maxit=60000, precond="aux")
    S0 = ref.sparams(r0)[f]
    Pm = problems.with_modal_ports(P, f)
    assert all(isinstance(p, ModalPort) for p in Pm.ports)
    beta = Pm.ports[0].get_beta(2 * np.pi * f / 299792458.0)
    assert abs(beta.real - P.ports[0].get_beta(2 * np.pi * f / 299792458.0)) < 3e-3 * beta.real
    sw = FrequencySweep(Pm)
    r1 = sw.solve([(f, 0), (f, 1)], tol=1e-10, maxit=60000, precond="aux")
    assert (r1.status == 0).all()
    S1 = sw.sparams(r1)[f]
    assert abs(abs(S1[1, 0]) - 1) < 0.01 and abs(S1[0, 0]) < 0.02
    assert np.abs(np.abs(S1) - np.abs(S0)).max() < 0.01
