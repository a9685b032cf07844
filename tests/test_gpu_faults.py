"""Host-injected faults come back as status codes / exceptions; no GPU fault, trap or hang.

Failures are made on the host (NaN tensors, a degenerate tet, out-of-range ids, an inconsistent
DOF map, an undersized workspace, an iteration cap of 1); the kernels' own checks turn them into
device status bits that the host reads."""
import ctypes

import numpy as np
import pytest
import torch

from emerge_b200 import _lib, assembly, problems
from emerge_b200._lib import EmfemError, Handle, lib, ptr
from emerge_b200.sweep import FrequencySweep

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prob():
    return problems.waveguide(nx=4, ny=2, nz=6, seed=2)


def _plan(P):
    dm = assembly.DeviceMesh(P.mesh, P.field)
    return dm, assembly.CsrPlan(dm)


def test_nan_material_reported(cuda, prob):
    dm, plan = _plan(prob)
    er = prob.er.copy()
    er[1, 1, 7] = np.nan
    plan.assemble(er, prob.ur)
    with pytest.raises(EmfemError, match="non-finite"):
        Handle.get().raise_on_device_status("nan test")
    # the context stays usable
    E, B = plan.assemble(prob.er, prob.ur)
    Handle.get().raise_on_device_status("clean run")
    assert torch.isfinite(torch.view_as_real(E)).all()


def test_degenerate_tet_reported(cuda, prob):
    nodes = prob.mesh.nodes.copy()
    t = prob.mesh.tets[:, 3]
    nodes[:, t[1]] = nodes[:, t[0]]        # collapse an edge of tet 3
    from emerge_b200.mesh import TetMesh
    from emerge_b200.nedelec2 import Nedelec2
    m = TetMesh(nodes, prob.mesh.tets)
    f = Nedelec2(m)
    with pytest.raises(EmfemError, match="degenerate"):
        assembly.tet_mass_stiffness_matrices(f, prob.er, prob.ur)


def test_out_of_range_node_id_reported(cuda, prob):
    dm, plan = _plan(prob)
    bad = dm.tets.clone()
    bad[2, 5] = dm.n_nodes + 100
    dm_tets = dm.tets
    dm.tets = bad
    try:
        plan.assemble(prob.er, prob.ur)
        with pytest.raises(EmfemError, match="index out of range"):
            Handle.get().raise_on_device_status("bad id")
    finally:
        dm.tets = dm_tets


def test_inconsistent_dof_map_rejected(cuda, prob):
    dm = assembly.DeviceMesh(prob.mesh, prob.field)
    dm.tet_to_field = dm.tet_to_field.clone()
    dm.tet_to_field[12, 0] += 1            # second-kind DOF no longer = first-kind + H
    with pytest.raises(EmfemError) as ei:
        assembly.CsrPlan(dm)
    assert ei.value.status == _lib.ERR_DEVICE_CHECK


def test_mesh_check_catches_wrong_edge_list(cuda, prob):
    import copy
    m = copy.copy(prob.mesh)
    m.edges = prob.mesh.edges.copy()
    m.edges[:, [3, 4]] = m.edges[:, [4, 3]]
    dm = assembly.DeviceMesh(m, prob.field)
    with pytest.raises(EmfemError, match="index out of range"):
        dm.check()


def test_undersized_workspace_and_bad_options(cuda, prob):
    sw = FrequencySweep(prob)
    b = sw.rhs([(10e9, 0)])
    x = torch.zeros_like(b)
    ws = torch.empty(1024, dtype=torch.uint8, device=b.device)
    st, it, rr = (ctypes.c_int * 1)(), (ctypes.c_int * 1)(), (ctypes.c_double * 1)()
    k0 = (ctypes.c_double * 1)(sw.k0sq([10e9])[0])
    g = sw.gammas([10e9])
    gam = (ctypes.c_double * 4)(*np.stack([g.real, g.imag], -1).ravel())
    h = Handle.get()
    args = lambda nsys, wsb: (h.h, 1, sw.n, sw.plan.nnz, ptr(sw.plan.indptr), ptr(sw.plan.indices), ptr(sw.E),
                              ptr(sw.B), nsys, k0, sw.patch_rows.numel(), ptr(sw.patch_rows), ptr(sw.patch_rowptr),
                              ptr(sw.patch_cols), ptr(sw.patch_vals), ptr(sw.patch_port), sw.n_ports, gam,
                              ptr(sw.mask), ptr(b), ptr(x), 1e-8, 100, 2, 0, ptr(ws), wsb, st, it, rr, None)
    assert lib().emfem_krylov_solve(*args(1, ws.numel())) == _lib.ERR_WORKSPACE
    assert "workspace" in _lib.last_error()
    assert lib().emfem_krylov_solve(*args(65, ws.numel())) == _lib.ERR_INVALID_ARG


def test_iteration_cap_reports_not_converged(cuda, prob):
    sw = FrequencySweep(prob)
    res = sw.solve([(10e9, 0), (10e9, 1)], tol=1e-12, maxit=3)
    assert (res.status == 1).all()
    assert (res.iters <= 4).all()
    assert np.isfinite(res.relres).all() and (res.relres > 1e-12).all()


def test_aux_preconditioner_misuse_is_rejected(cuda, prob):
    """The aux-space and learned preconditioners refuse to run without their set-up, and a bad
    edge list is caught by the device check, all as status codes."""
    sw = FrequencySweep(prob)
    b = sw.rhs([(10e9, 0)])
    x = torch.zeros_like(b)
    sz = ctypes.c_size_t()
    lib().emfem_krylov_workspace_size(sw.n, sw.plan.nnz, 1, 0, ctypes.byref(sz))
    ws = torch.empty(sz.value, dtype=torch.uint8, device=b.device)
    st, it, rr = (ctypes.c_int * 1)(), (ctypes.c_int * 1)(), (ctypes.c_double * 1)()
    k0 = (ctypes.c_double * 1)(sw.k0sq([10e9])[0])
    g = sw.gammas([10e9])
    gam = (ctypes.c_double * 4)(*np.stack([g.real, g.imag], -1).ravel())
    h = Handle.get()

    def call(precond, method, aux):
        return lib().emfem_krylov_solve(h.h, method, sw.n, sw.plan.nnz, ptr(sw.plan.indptr), ptr(sw.plan.indices),
                                        ptr(sw.E), ptr(sw.B), 1, k0, sw.patch_rows.numel(), ptr(sw.patch_rows),
                                        ptr(sw.patch_rowptr), ptr(sw.patch_cols), ptr(sw.patch_vals),
                                        ptr(sw.patch_port), sw.n_ports, gam, ptr(sw.mask), ptr(b), ptr(x), 1e-8, 50,
                                        precond, 0, ptr(ws), ws.numel(), st, it, rr, aux)

    assert call(3, 1, None) == _lib.ERR_INVALID_ARG              # no aux space
    from emerge_b200.auxspace import AuxSpace
    aux = AuxSpace(prob.mesh)
    assert call(3, 1, aux.handle) == _lib.ERR_INVALID_ARG        # no operator set yet
    aux.set_operator(sw)
    assert call(3, 1, aux.handle) == _lib.ERR_INVALID_ARG        # buffers not reserved
    aux.reserve(1)
    assert call(3, 0, aux.handle) == _lib.ERR_INVALID_ARG        # COCG with the aux correction
    assert call(4, 1, aux.handle) == _lib.ERR_INVALID_ARG        # learned without parameters
    assert call(3, 1, aux.handle) in (0, _lib.ERR_NOT_CONVERGED)  # properly set up: runs
    # an edge with an out-of-range node id is caught by the device check
    bad = prob.mesh.edges.copy()
    bad[1, 3] = prob.mesh.n_nodes + 7

    class M:
        nodes, edges, tris = prob.mesh.nodes, bad, prob.mesh.tris
        tri_to_edge, edge_lengths = prob.mesh.tri_to_edge, prob.mesh.edge_lengths
    with pytest.raises(EmfemError):
        AuxSpace(M)
    AuxSpace(prob.mesh)                                           # the handle stays usable
