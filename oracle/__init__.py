"""CPU oracle for the Nédélec-2 hot path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
this package, always as the checker and never as the measured or shipped path.

* ``libned2_oracle.so`` (built from ``ned2_oracle.c`` by ``oracle/Makefile``) restates the reference's
  numba kernels: ``_matrix_builder`` / ``ned2_tet_stiff_mass`` (``ASM/curlcurl.py:180-466``) and the
  Robin triangle kernels (``ASM/robinbc.py:126-443``).
* This module wraps it with the reference's Python signatures and adds the SciPy steps the
  reference performs around the kernels: COO→CSR with duplicate summation (``ASM/curlcurl.py:170-171``),
  ``K = E − k0²·B`` (``ASM/assembler.py:255``), ``generate_csr`` (``elements/femdata.py:131-134``) and
  the SuperLU direct solve of ``SolverSuperLU`` through ``SolveRoutine.solve``
  (``solver.py:561-572``, ``:1266-1313``).

Pinned against golden vectors produced by the reference itself (``tests/golden/make_golden.py``;
checked by ``tests/test_oracle_golden.py``).

``ASM/`` = ``src/emerge/_emerge/physics/microwave/assembly/``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
from scipy.sparse import coo_matrix, csr_matrix
from scipy.sparse.linalg import splu

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "libned2_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int64)


def build(force: bool = False) -> str:
    """Compile ``libned2_oracle.so`` with the system gcc (OpenMP)."""
    if force or not os.path.exists(_LIBPATH) or \
            os.path.getmtime(_LIBPATH) < os.path.getmtime(os.path.join(_HERE, "ned2_oracle.c")):
        subprocess.run(["make", "-s", "-C", _HERE, "ORACLE_CC=gcc"], check=True)
    return _LIBPATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIBPATH):
            build()
        L = ctypes.CDLL(_LIBPATH)
        L.oracle_matrix_builder.argtypes = [ctypes.c_int64] * 4 + [_dp, _ip, _ip, _ip, _dp, _ip, _ip, _dp, _dp, _dp, _dp, _ip, _ip]
        L.oracle_matrix_builder.restype = None
        L.oracle_robin_entries.argtypes = [ctypes.c_int64, ctypes.c_int64, _dp, _ip, _ip, ctypes.c_int64,
                                           ctypes.c_double, ctypes.c_double, _dp, _dp, ctypes.c_int, _ip, _dp, _dp]
        L.oracle_robin_entries.restype = None
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_set_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return lib().oracle_set_threads(int(n))


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    return a.ctypes.data_as(_dp if a.dtype in (np.float64, np.complex128) else _ip)


def _cplx(z: complex):
    return complex(z).real, complex(z).imag


# ------------------------------------------------------------------ tet path
def matrix_builder(nodes, tets, tris, edges, all_edge_lengths, tet_to_field, tet_to_edge, ur, er):
    """``_matrix_builder`` (ASM/curlcurl.py:419-466): (dataE, dataB, rows, cols), 400 entries per tet."""
    nodes = _c(nodes, np.float64); tets = _c(tets, np.int64); tris = _c(tris, np.int64)
    edges = _c(edges, np.int64); el = _c(all_edge_lengths, np.float64)
    t2f = _c(tet_to_field, np.int64); t2e = _c(tet_to_edge, np.int64)
    ur = _c(ur, np.complex128); er = _c(er, np.complex128)
    nt = tets.shape[1]
    dataE = np.empty(400 * nt, np.complex128); dataB = np.empty(400 * nt, np.complex128)
    rows = np.empty(400 * nt, np.int64); cols = np.empty(400 * nt, np.int64)
    lib().oracle_matrix_builder(nodes.shape[1], nt, tris.shape[1], edges.shape[1], _p(nodes), _p(tets), _p(tris),
                                _p(edges), _p(el), _p(t2f), _p(t2e), _p(ur), _p(er),
                                _p(dataE), _p(dataB), _p(rows), _p(cols))
    return dataE, dataB, rows, cols


def tet_mass_stiffness_matrices(field, er, ur) -> tuple[csr_matrix, csr_matrix]:
    """``tet_mass_stiffness_matrices`` (ASM/curlcurl.py:145-173): E (curl-curl) and B (mass) CSR."""
    m = field.mesh
    dataE, dataB, rows, cols = matrix_builder(m.nodes, m.tets, m.tris, m.edges, m.edge_lengths,
                                              field.tet_to_field, m.tet_to_edge, ur, er)
    n = 2 * m.n_edges + 2 * m.n_tris
    E = coo_matrix((dataE, (rows, cols)), shape=(n, n)).tocsr()
    B = coo_matrix((dataB, (rows, cols)), shape=(n, n)).tocsr()
    return E, B


# ------------------------------------------------------------------ Robin / port path
def dunavant4() -> np.ndarray:
    """Dunavant's degree-4, 6-point triangle rule as (4, 6) [W, L1, L2, L3] in the point order of
    ``gaus_quad_tri(4)`` (mth/optimized.py:87-118)."""
    pts = []
    for w, l1, l2, l3 in ((0.223381589678011, 0.108103018168070, 0.445948490915965, 0.445948490915965),
                          (0.109951743655322, 0.816847572980459, 0.091576213509771, 0.091576213509771)):
        a, b, c = l1, l2, l3
        for _ in range(3):
            pts.append([w, a, b, c])
            a, b, c = b, c, a
    return np.array(pts, dtype=np.float64).T.copy()


def generate_points_3d(nodes, tris, DPTs, tri_ids):
    """Quadrature points of the listed triangles, flattened point-major (robinbc.py:91-111)."""
    v = nodes[:, tris[:, tri_ids]]                       # (3, 3, ns)
    pts = np.einsum("cvs,vp->cps", v, DPTs[1:4])         # (3, npts, ns)
    return pts[0].ravel(), pts[1].ravel(), pts[2].ravel()


def _robin(field, Bmat, tri_ids, gamma, U, DPTs, Bvec):
    m = field.mesh
    tri_ids = _c(tri_ids, np.int64)
    nodes = _c(m.nodes, np.float64); tris = _c(m.tris, np.int64)
    t2f = _c(field.tri_to_field, np.int64)
    dpts = _c(DPTs if DPTs is not None else dunavant4(), np.float64)
    assert Bmat.dtype == np.complex128 and Bmat.flags.c_contiguous
    Up = None if U is None else _p(U)
    lib().oracle_robin_entries(nodes.shape[1], tris.shape[1], _p(nodes), _p(tris), _p(tri_ids), len(tri_ids),
                               *_cplx(gamma), Up, _p(dpts), dpts.shape[1], _p(t2f), _p(Bmat),
                               None if Bvec is None else _p(Bvec))


def assemble_robin_bc_excited(field, Bmat, surf_triangle_indices, Ufunc, gamma, DPTs):
    """``assemble_robin_bc_excited`` (robinbc.py:445-463); Bmat is updated in place and returned."""
    Bvec = np.zeros(field.n_field, dtype=np.complex128)
    x, y, z = generate_points_3d(field.mesh.nodes, field.mesh.tris, DPTs, surf_triangle_indices)
    U = np.asarray(Ufunc(x, y, z), dtype=np.complex128).reshape(3, DPTs.shape[1], len(surf_triangle_indices))
    U = np.ascontiguousarray(U)
    _robin(field, Bmat, surf_triangle_indices, gamma, U, DPTs, Bvec)
    return Bmat, Bvec


def assemble_robin_bc(field, Bmat, surf_triangle_indices, gamma):
    """``assemble_robin_bc`` (robinbc.py:465-473); Bmat is updated in place and returned."""
    _robin(field, Bmat, surf_triangle_indices, gamma, None, None, None)
    return Bmat


# ------------------------------------------------------------------ direct solve
def superlu_factor(A, pivoting_threshold: float = 0.001):
    """The factorisation of ``SolverSuperLU.solve`` (solver.py:561-572)."""
    lu = splu(A.tocsc(), permc_spec="MMD_AT_PLUS_A", relax=0, diag_pivot_thresh=pivoting_threshold,
              options=dict(SymmetricMode=True, Equil=False, IterRefine="SINGLE"))
    return lu


def solve_routine(A, rhs_list, solve_ids):
    """``SolveRoutine.solve`` (solver.py:1241-1326) for several right-hand sides sharing one LU:
    PEC DOFs eliminated by submatrix, SuperLU, scatter back with zeros on eliminated DOFs."""
    n = A.shape[0]
    Asel = A.tocsc()[np.ix_(solve_ids, solve_ids)]
    lu = superlu_factor(Asel)
    out = []
    for b in rhs_list:
        x = np.zeros(n, dtype=np.complex128)
        x[solve_ids] = lu.solve(np.asarray(b)[solve_ids])
        out.append(x)
    return out
