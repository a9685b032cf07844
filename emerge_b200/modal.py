"""Port-mode (boundary-mode) analysis: the 2-D eigenproblem of a port face, assembled on the device.

The reference finds the modes of a ``ModalPort`` by ``Microwave3D.modal_analysis``
(``MW/microwave_3d.py:474-650``): ``Assembler.assemble_bma_matrices`` (``ASM/assembler.py:110-187``)
cuts the port face out of the mesh as a ``SurfaceMesh`` (``mesh3d.py:717-880``), numbers a
``NedelecLegrange2`` field on it (``elements/nedleg2.py:102-166``), builds the element matrices with
``generelized_eigenvalue_matrix`` (``ASM/generalized_eigen_hb.py:41-62, 257-458``) and removes PEC DOFs;
``SolveRoutine.eig_boundary`` (``solver.py:1328-1374``) then solves A e = -beta^2 B e with dense LAPACK
(``SolverLAPACK``, :780-810, below 1000 DOFs or when ``direct``) or shift-invert ARPACK.

Here the triangle blocks come from ``emfem_ned2_bma_tri_matrices`` (one device launch for the whole
face) and are summed into CSR slots on the device (``emfem_segmented_gather_sum``); the eigen-solve of
the small reduced system stays with LAPACK/ARPACK on the host, as in the reference.

Differences in numbering only: :class:`PortSurface` lists the face's edges in lexicographic order of
their (min, max) node ids, where ``SurfaceMesh`` keeps Python ``set`` order.  Nodes and triangles are in
the reference's order; the matrices are the same up to that permutation of edge DOFs.

``ASM/`` = ``src/emerge/_emerge/physics/microwave/assembly/``; ``MW/`` = ``src/emerge/_emerge/physics/microwave/``.
"""
from __future__ import annotations

from dataclasses import dataclass, field as dfield

import numpy as np
import scipy.linalg
import scipy.sparse.linalg
import torch
from scipy.sparse import csr_matrix

from ._lib import Handle, check, lib, ptr
from .assembly import _device, _to_dev, dunavant4
from .constants import C0, EPS0, MU0
from .ports import PortFrame

__all__ = ["PortFrame", "PortSurface", "NedLeg2Field", "PortMode", "bma_blocks", "assemble_bma_matrices",
           "eig_boundary", "modal_analysis", "tri_field", "mode_fields_global", "mode_power", "face_normal",
           "PEC_CONDUCTIVITY"]

PEC_CONDUCTIVITY = 1e7        # Settings.mw_3d_peclim default (settings.py:24)


class PortSurface:
    """The port face as a 2-D mesh (``SurfaceMesh``, ``mesh3d.py:717-880``).

    ``tri_ids`` index the 3-D mesh's triangles; nodes are the sorted unique node ids of those triangles,
    triangles keep their order and (sorted) vertex order, edges are the unique (min, max) pairs sorted
    lexicographically, ``tri_to_edge`` = [e(v1, v2), e(v2, v3), e(v1, v3)] (:866-872)."""

    def __init__(self, mesh, tri_ids, frame: PortFrame):
        self.tri_ids = np.asarray(tri_ids, dtype=np.int64)
        if self.tri_ids.size == 0:
            raise ValueError("PortSurface: no triangles")
        t3 = np.asarray(mesh.tris)[:, self.tri_ids]
        self.node_ids = np.unique(t3)
        self.tris = np.searchsorted(self.node_ids, t3).astype(np.int64)
        self.nodes = np.asarray(mesh.nodes)[:, self.node_ids]
        nn = self.node_ids.size
        pairs = [(self.tris[p], self.tris[q]) for p, q in ((0, 1), (1, 2), (0, 2))]
        keys = [np.minimum(u, v) * nn + np.maximum(u, v) for u, v in pairs]
        ukeys = np.unique(np.concatenate(keys))
        self.edges = np.stack([ukeys // nn, ukeys % nn]).astype(np.int64)
        self.tri_to_edge = np.stack([np.searchsorted(ukeys, k) for k in keys]).astype(np.int64)
        self._ekeys = ukeys
        self.frame = frame
        self.local_nodes = frame.in_local_cs(self.nodes)

    @property
    def n_nodes(self) -> int:
        return self.nodes.shape[1]

    @property
    def n_edges(self) -> int:
        return self.edges.shape[1]

    @property
    def n_tris(self) -> int:
        return self.tris.shape[1]

    def from_source_edges(self, edges3d: np.ndarray) -> np.ndarray:
        """Surface edge ids of 3-D edges given as (2, k) global node pairs; -1 where an edge is not on
        the face (``SurfaceMesh.from_source_edge``, :799-805)."""
        e = np.asarray(edges3d, dtype=np.int64)
        loc = np.searchsorted(self.node_ids, e)
        loc = np.minimum(loc, self.node_ids.size - 1)
        on = (self.node_ids[loc] == e).all(axis=0)
        nn = self.node_ids.size
        key = np.minimum(loc[0], loc[1]) * nn + np.maximum(loc[0], loc[1])
        pos = np.minimum(np.searchsorted(self._ekeys, key), self._ekeys.size - 1)
        hit = on & (self._ekeys[pos] == key)
        return np.where(hit, pos, -1)


class NedLeg2Field:
    """DOF numbering of ``NedelecLegrange2`` (``elements/nedleg2.py:102-166``) with Lagrange order 2:
    [edges | faces | edges' | faces' | vertices (E_z) | edge midpoints (E_z)]."""

    def __init__(self, surface: PortSurface):
        Nn, Ne, Nt = surface.n_nodes, surface.n_edges, surface.n_tris
        self.mesh = surface
        self.n_field = 2 * Ne + 2 * Nt + Nn + Ne
        self.n_xy = 2 * Ne + 2 * Nt
        t2f = np.zeros((14, Nt), dtype=np.int64)
        t2f[:3] = surface.tri_to_edge
        t2f[3] = np.arange(Nt) + Ne
        t2f[4:7] = surface.tri_to_edge + Ne + Nt
        t2f[7] = np.arange(Nt) + 2 * Ne + Nt
        t2f[8:11] = surface.tris + 2 * Ne + 2 * Nt
        t2f[11:14] = surface.tri_to_edge + 2 * Ne + 2 * Nt + Nn
        self.tri_to_field = t2f
        e2f = np.zeros((5, Ne), dtype=np.int64)
        e2f[0] = np.arange(Ne)
        e2f[1] = np.arange(Ne) + Nt + Ne
        e2f[2:4] = surface.edges + 2 * Ne + 2 * Nt
        e2f[4] = np.arange(Ne) + 2 * Ne + 2 * Nt + Nn
        self.edge_to_field = e2f


def bma_blocks(surface: PortSurface, er: np.ndarray, ur: np.ndarray, k0: float, device=None):
    """(A, B) (n_tris, 196) complex128 device tensors: the reference's dataE / dataB per triangle."""
    dev = _device(device)
    nt = surface.n_tris
    er = _to_dev(np.asarray(er, dtype=np.complex128).reshape(9, nt), torch.complex128, dev)
    ur = _to_dev(np.asarray(ur, dtype=np.complex128).reshape(9, nt), torch.complex128, dev)
    ln = _to_dev(surface.local_nodes[:2], torch.float64, dev)
    tris = _to_dev(surface.tris, torch.int64, dev)
    edges = _to_dev(surface.edges, torch.int64, dev)
    t2e = _to_dev(surface.tri_to_edge, torch.int64, dev)
    A = torch.empty((nt, 196), dtype=torch.complex128, device=dev)
    B = torch.empty_like(A)
    h = Handle.get(dev)
    check(lib().emfem_ned2_bma_tri_matrices(h.h, surface.n_nodes, ptr(ln), nt, ptr(tris), surface.n_edges,
                                            ptr(edges), ptr(t2e), ptr(er), ptr(ur), float(k0), ptr(A), ptr(B)),
          "emfem_ned2_bma_tri_matrices")
    h.raise_on_device_status("emfem_ned2_bma_tri_matrices")
    return A, B


def _csr(field: NedLeg2Field, A: torch.Tensor, B: torch.Tensor):
    """COO -> CSR with duplicate summation (``generelized_eigenvalue_matrix``, :56-59), values summed on
    the device in triangle order per slot."""
    from .sweep import _seg_from_keys, gather_sum
    n = field.n_field
    idx = field.tri_to_field.T                                   # (nt, 14)
    rows = np.repeat(idx, 14, axis=1).ravel()
    cols = np.tile(idx, (1, 14)).ravel()
    ukeys, seg, order = _seg_from_keys(rows * n + cols)
    dev = A.device
    seg_d = torch.from_numpy(seg).to(dev)
    ord_d = torch.from_numpy(order).to(dev)
    ev = gather_sum(seg_d, ord_d, A.reshape(-1)).cpu().numpy()
    bv = gather_sum(seg_d, ord_d, B.reshape(-1)).cpu().numpy()
    r, c = ukeys // n, ukeys % n
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(indptr, r + 1, 1)
    indptr = np.cumsum(indptr).astype(np.int32)
    cc = c.astype(np.int32)
    return csr_matrix((ev, cc, indptr), shape=(n, n)), csr_matrix((bv, cc.copy(), indptr.copy()), shape=(n, n))


def assemble_bma_matrices(mesh, tri_ids, frame: PortFrame, er, ur, k0: float, sig=None, pec_edges=None,
                          peclim: float = PEC_CONDUCTIVITY, device=None):
    """Drop-in for ``Assembler.assemble_bma_matrices`` (``ASM/assembler.py:110-187``).

    er, ur: (3, 3, n_sel) complex material tensors of the port triangles (the reference's
    ``er[:, :, tri_ids]``); sig: (n_sel,) conductivity or None, added as er - j sig/(k0 c0 eps0) and
    turning a triangle into PEC above ``peclim``; pec_edges: (2, k) global node pairs of edges on PEC
    boundaries (the edges of the PEC faces' triangles).  Returns (E, B, solve_ids, field) with E, B
    SciPy CSR matrices on the host."""
    surf = PortSurface(mesh, tri_ids, frame)
    fld = NedLeg2Field(surf)
    er = np.asarray(er, dtype=np.complex128)
    ur = np.asarray(ur, dtype=np.complex128)
    sig = np.zeros(surf.n_tris) if sig is None else np.asarray(sig, dtype=np.float64)
    er = er - 1j * sig / (k0 * C0 * EPS0)
    A, B = bma_blocks(surf, er, ur, k0, device)
    E, Bm = _csr(fld, A, B)
    pec = np.zeros(fld.n_field, dtype=bool)
    pec[fld.tri_to_field[:, sig > peclim].ravel()] = True
    if pec_edges is not None and np.size(pec_edges):
        se = surf.from_source_edges(pec_edges)
        se = se[se >= 0]
        pec[fld.edge_to_field[:, se].ravel()] = True
    solve_ids = np.flatnonzero(~pec).astype(np.int64)
    return E, Bm, solve_ids, fld


def _filter_real_modes(lam, vecs, k0, ermax, urmax, sign):
    """``filter_real_modes`` (``solver.py:192-227``): keep sign*lambda in [1, 2 k0^2 er ur], ascending |beta|."""
    ext = (k0 ** 2) * ermax * urmax * 2
    mask = (sign * lam <= ext) & (sign * lam >= 1)
    lam, vecs = lam[mask], vecs[:, mask]
    order = np.argsort(np.abs(np.sqrt(sign * lam)))
    return lam[order], vecs[:, order]


def eig_boundary(E: csr_matrix, B: csr_matrix, solve_ids: np.ndarray, nmodes: int = 6, direct: bool = True,
                 target_kz: float = 0.0, sign: float = -1.0):
    """Eigenpairs of E x = lambda B x on the free DOFs (``SolveRoutine.eig_boundary``, ``solver.py:1328-1374``).

    Dense LAPACK below 1000 DOFs or when ``direct`` (``SolverLAPACK.eig``, :780-810, whose filter takes
    er = ur = 2); otherwise one shift-invert ARPACK solve at sigma = sign target_kz^2 for ``nmodes``
    pairs.  (The reference's ``SmartARPACK_BMA``, :832-878, repeats single-pair solves over 81 shifts
    around the target and keeps the most energetic; both return the modes nearest the target.)"""
    Asel = E[np.ix_(solve_ids, solve_ids)]
    Bsel = B[np.ix_(solve_ids, solve_ids)]
    if direct or Asel.shape[0] < 1000:
        lam, vecs = scipy.linalg.eig(Asel.toarray(), Bsel.toarray(), overwrite_a=True, overwrite_b=True,
                                     check_finite=False)
        return _filter_real_modes(lam, vecs, target_kz, 2, 2, sign)
    lam, vecs = scipy.sparse.linalg.eigs(Asel.tocsc(), k=nmodes, M=Bsel.tocsc(), sigma=sign * target_kz ** 2,
                                         which="LM")
    return lam, vecs


@dataclass
class PortMode:
    """One port mode (``PortMode``, ``MW/microwave_bc.py:347-372``)."""
    modefield: np.ndarray
    k0: float
    beta: complex
    freq: float
    modetype: str = "TE"
    polarity: float = 1.0
    norm_factor: float = 1.0
    power: float = 0.0
    energy: float = dfield(init=False)
    neff: complex = dfield(init=False)

    def __post_init__(self):
        self.neff = self.beta / self.k0
        self.energy = float(np.mean(np.abs(self.modefield) ** 2))


def modal_analysis(mesh, tri_ids, frame: PortFrame, er, ur, freq: float, nmodes: int = 6, direct: bool = True,
                   TEM: bool = False, target_kz: float | None = None, target_neff: float | None = None,
                   sig=None, pec_edges=None, device=None, sort: bool = True):
    """Modes of a port face (``Microwave3D.modal_analysis``, ``MW/microwave_3d.py:474-650``).

    Returns the modes sorted by descending beta (``ModalPort.sort_modes``, ``MW/microwave_bc.py:613-637``,
    without alignment vectors).  Each mode's field is the full NedelecLegrange2 vector (zeros on PEC
    DOFs) rotated so its largest entry is real (:581-584); beta = min(k0 sqrt(er_max ur_max), sqrt(-lambda))
    (:587-588); a mode whose mean |e|^2 is below 1e-4 is dropped (``ModalPort.add_mode``, :688-690);
    the type is TE when max|E_z| / max|E_t| < 0.1, else TM, or TEM when asked (:622-646).  With
    ``sort=False`` the modes stay in the eigen-solver's order (ascending |beta| for LAPACK)."""
    k0 = 2 * np.pi * freq / C0
    er = np.asarray(er, dtype=np.complex128)
    ur = np.asarray(ur, dtype=np.complex128)
    E, B, solve_ids, fld = assemble_bma_matrices(mesh, tri_ids, frame, er, ur, k0, sig, pec_edges, device=device)
    dg_e = np.real(np.diagonal(er, axis1=0, axis2=1))
    dg_u = np.real(np.diagonal(ur, axis1=0, axis2=1))
    ermean, urmean = float(np.mean(dg_e[dg_e > 0])), float(np.mean(dg_u[dg_u > 0]))
    ermax, urmax = np.max(er), np.max(ur)
    if target_neff is not None:
        target_kz = k0 * target_neff
    if target_kz is None:
        target_kz = ermean * urmean * (1.1 if TEM else 0.7) * k0
    lam, vecs = eig_boundary(E, B, solve_ids, nmodes, direct, target_kz, sign=-1.0)
    modes = []
    for i in range(lam.shape[0]):
        em = np.zeros(fld.n_field, dtype=np.complex128)
        em[solve_ids] = vecs[:, i]
        em = em * np.exp(-1j * np.angle(em[np.argmax(np.abs(em))]))
        beta_base = np.emath.sqrt(-lam[i])
        cap = k0 * np.sqrt(ermax * urmax)
        beta = cap if (np.real(cap), np.imag(cap)) < (np.real(beta_base), np.imag(beta_base)) else beta_base
        if TEM:
            mt = "TEM"
        else:
            ez, exy = np.max(np.abs(em[fld.n_xy:])), np.max(np.abs(em[:fld.n_xy]))
            mt = "TE" if ez / exy < 1e-1 else "TM"
        m = PortMode(em, k0, complex(beta), freq, mt)
        if m.energy < 1e-4:
            continue
        modes.append(m)
    if sort:
        modes.sort(key=lambda m: m.beta.real, reverse=True)
    return modes, fld


def _local_points(surface: PortSurface, pts: np.ndarray) -> np.ndarray:
    """Global points (3, npts, n_tris), column t inside face triangle t -> local (2, npts, n_tris);
    raises when a point lies outside its triangle (barycentric test of ``ned2_tri_interp_full``)."""
    npts, nt = pts.shape[1], pts.shape[2]
    if nt != surface.n_tris:
        raise ValueError("points must be given per face triangle: (3, npts, n_tris)")
    loc = surface.frame.in_local_cs(pts.reshape(3, -1)).reshape(3, npts, nt)[:2]
    v = surface.local_nodes[:2][:, surface.tris]                      # (2, 3, nt)
    e1, e2 = v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]
    det = e1[0] * e2[1] - e1[1] * e2[0]
    d = loc - v[:, 0][:, None, :]
    u = (d[0] * e2[1] - d[1] * e2[0]) / det
    w = (e1[0] * d[1] - e1[1] * d[0]) / det
    if not ((u >= -1e-6) & (w >= -1e-6) & (u + w <= 1.00001)).all():
        raise ValueError("a point lies outside its face triangle")
    return np.ascontiguousarray(loc)


def tri_field(surface: PortSurface, field: NedLeg2Field, x, pts_local: np.ndarray, what: str = "E",
              beta: complex = 0.0, diadic=None, device=None) -> torch.Tensor:
    """(3, npts, n_tris) complex field of the mode vector x in the port's local frame at per-triangle
    local points: E, or for ``what="H"`` the curl form of ``ned2_tri_interp_curl`` times the diagonal of
    ``diadic`` (3, n_tris) (without the factor j/(k0 c0 mu0))."""
    dev = _device(device)
    npts, nt = pts_local.shape[1], pts_local.shape[2]
    xd = _to_dev(np.asarray(x, dtype=np.complex128), torch.complex128, dev)
    pd = _to_dev(pts_local, torch.float64, dev)
    ln = _to_dev(surface.local_nodes[:2], torch.float64, dev)
    tris = _to_dev(surface.tris, torch.int64, dev)
    edges = _to_dev(surface.edges, torch.int64, dev)
    t2e = _to_dev(surface.tri_to_edge, torch.int64, dev)
    t2f = _to_dev(field.tri_to_field, torch.int64, dev)
    dg = None if diadic is None else _to_dev(np.asarray(diadic, dtype=np.complex128).reshape(3, nt),
                                             torch.complex128, dev)
    out = torch.empty((3, npts, nt), dtype=torch.complex128, device=dev)
    b = complex(beta)
    h = Handle.get(dev)
    check(lib().emfem_ned2_tri_field(h.h, surface.n_nodes, ptr(ln), nt, ptr(tris), surface.n_edges, ptr(edges),
                                     ptr(t2e), ptr(t2f), field.n_field, ptr(xd), npts, ptr(pd),
                                     0 if what == "E" else 1, b.real, b.imag, None if dg is None else ptr(dg),
                                     ptr(out)), "emfem_ned2_tri_field")
    h.raise_on_device_status("emfem_ned2_tri_field")
    return out


def mode_fields_global(surface, field, x, pts, k0=None, ur=None, beta=0.0, device=None):
    """E (and, with k0 and ur, H) of a mode at per-triangle global points (3, npts, n_tris), global basis
    (``FieldFunctionClass.__call__``, ``elements/nedleg2.py:62-72``; H = j/(k0 c0 mu0) ur^-1 curl E)."""
    loc = _local_points(surface, np.asarray(pts, dtype=np.float64))
    fr = surface.frame
    E = tri_field(surface, field, x, loc, "E", device=device).cpu().numpy()
    Eg = fr.in_global_basis(E.reshape(3, -1)).reshape(E.shape)
    if k0 is None:
        return Eg
    urinv = _diag_inv(ur)
    H = tri_field(surface, field, x, loc, "H", beta, urinv, device=device).cpu().numpy()
    H = H * (1j / (k0 * C0 * MU0))
    return Eg, fr.in_global_basis(H.reshape(3, -1)).reshape(H.shape)


def _diag_inv(ur) -> np.ndarray:
    """Diagonal (3, n) of ur^-1 per triangle: the diadic of ``interpolate_Hf`` (``elements/nedleg2.py:
    172-180``), inverted like ``matinv`` (``mth/optimized.py:342-370``: 1/diagonal when off-diagonals
    vanish); ``ned2_tri_interp_curl`` only uses the diagonal."""
    ur = np.asarray(ur, dtype=np.complex128)
    n = ur.shape[2]
    out = np.zeros((3, n), dtype=np.complex128)
    off = np.zeros(n, dtype=bool)
    for i in range(3):
        for j in range(3):
            if i != j:
                off |= ur[i, j] != 0
    for i in range(3):
        out[i, ~off] = 1.0 / ur[i, i, ~off]
    if off.any():
        inv = np.linalg.inv(ur[:, :, off].transpose(2, 0, 1))
        out[:, off] = np.stack([inv[:, i, i] for i in range(3)])
    return out


def face_normal(surface: PortSurface) -> np.ndarray:
    """Unit normal of the face's first triangle pointing away from origin - z_axis of the port frame
    (``SurfaceMesh`` normals via ``outward_normal``, ``mth/optimized.py:252-274``, with the alignment
    origin of ``assemble_bma_matrices``, ``ASM/assembler.py:141``)."""
    n1, n2, n3 = (surface.nodes[:, surface.tris[k, 0]] for k in range(3))
    n = np.cross(n2 - n1, n3 - n1)
    n = n / np.sqrt(n @ n)
    o = surface.frame.origin - surface.frame.basis[:, 2]
    return -n if n @ ((n1 + n2 + n3) / 3.0 - o) < 0 else n


def mode_power(surface: PortSurface, field: NedLeg2Field, x, k0: float, ur, beta, device=None) -> float:
    """Average power flux of a mode through the face, integral of 1/2 Re(E x H*) . n with the order-4
    Dunavant rule (``compute_avg_power_flux``, ``MW/port_functions.py:21-36``, ``surface_integral``
    ``mth/integrals.py:60-100``)."""
    dp = dunavant4()
    v = surface.nodes[:, surface.tris]                                   # (3, 3, nt)
    pts = np.einsum("cvs,vp->cps", v, dp[1:4])
    E, H = mode_fields_global(surface, field, x, pts, k0, ur, beta, device)
    nrm = face_normal(surface)
    Hc = np.conj(H)
    Sx = 0.5 * np.real(E[1] * Hc[2] - E[2] * Hc[1])
    Sy = 0.5 * np.real(E[2] * Hc[0] - E[0] * Hc[2])
    Sz = 0.5 * np.real(E[0] * Hc[1] - E[1] * Hc[0])
    S = nrm[0] * Sx + nrm[1] * Sy + nrm[2] * Sz                         # (npts, nt)
    cr = np.cross((v[:, 1] - v[:, 0]).T, (v[:, 2] - v[:, 0]).T)
    area = np.sqrt(np.sum(cr ** 2, axis=1)) / 2
    return float(np.sum(area * np.sum(dp[0][:, None] * S, axis=0)))
