"""Frequency-domain assembly with the flow of ``Assembler.assemble_freq_matrix``
(``src/emerge/_emerge/physics/microwave/assembly/assembler.py:189-429``) and the ``SimJob`` it
returns (``src/emerge/_emerge/physics/microwave/simjob.py:23-136``).

Material tensors are passed in directly as (3, 3, N_t) εr/μr arrays (the reference derives them
from ``emsutil.Material`` objects with ``er·(1−j·tanδ) − j·σ/(ωε0)``, ``assembler.py:229-240``);
ports are :class:`~emerge_b200.ports.RectangularWaveguidePort` objects; PEC is a list of boundary
triangles.  Everything the reference computes on the matrices runs on the GPU: E and B (kept on the
device between frequencies when ``cache_matrices``), the Robin/port triangle blocks summed per
triangle as the reference's ``Bempty`` (``:314-347``) and per CSR slot as ``generate_csr``
(``elements/femdata.py:131-134``), ``K = E − B·K0² + B_p`` (``:255``, ``:350``) and the removal of the
exact zeros that SciPy's sparse arithmetic leaves out.  Only K crosses to the host.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
from scipy.sparse import csr_matrix

from ._lib import Handle, check, lib, ptr
from .assembly import _device, _plan_for, dunavant4, tri_abc2_device, tri_robin_device
from .ports import k0_of
from .sweep import _seg_from_keys, gather_sum


class SimJob:
    def __init__(self, A, b, freq: float, cache_factorization: bool = True):
        self.A = A
        self.b = b
        self.freq = freq
        self.k0 = 2 * np.pi * freq / 299792458
        self.cache_factorization = cache_factorization
        self._fields: dict[int, np.ndarray] = {}
        self.port_vectors: dict[int, np.ndarray] | None = None
        self.solve_ids: np.ndarray | None = None
        self._active_port = -1
        self.reports = []

    def iter_Ab(self):
        """One (A, b + port vector) per port; the factorization is reused after the first (simjob.py:82-107)."""
        reuse = False
        for key, mode in self.port_vectors.items():
            self._active_port = key
            yield self.A, self.b + mode, self.solve_ids, reuse, {"Active port": str(key)}
            reuse = True

    def submit_solution(self, solution: np.ndarray, report) -> None:
        self._fields[self._active_port] = solution
        self.reports.append(report)


class Assembler:
    def __init__(self):
        self.cached_matrices = None       # (plan, E, B): device values on the field's plan

    def assemble_freq_matrix(self, field, er: np.ndarray, ur: np.ndarray, ports, pec_tris: np.ndarray,
                             frequency: float, cache_matrices: bool = False, device=None, robin_bcs=()) -> SimJob:
        dev = _device(device)
        dm, plan = _plan_for(field, dev)
        K0 = k0_of(frequency)
        h = Handle.get(dev)
        if cache_matrices and self.cached_matrices is not None and self.cached_matrices[0] is plan:
            _, E, B = self.cached_matrices
        else:
            E, B = plan.assemble(er, ur)
            h.raise_on_device_status("assemble_freq_matrix")
            self.cached_matrices = (plan, E, B)
        N = field.n_field
        b = np.zeros(N, dtype=np.complex128)
        port_vectors = {p.port_number: np.zeros(N, dtype=np.complex128) for p in ports}
        pec_ids = field.pec_dofs(pec_tris) if len(pec_tris) else np.zeros(0, dtype=np.int64)
        slots = vals = None
        if len(ports) or len(robin_bcs):
            slots, vals = self._robin_patch(field, dm, plan, ports, robin_bcs, K0, port_vectors)
        K = freq_matrix_device(plan, E, B, K0 ** 2, slots, vals)
        job = SimJob(K, b, K0 * 299792458 / (2 * np.pi), True)
        job.port_vectors = port_vectors
        job.solve_ids = field.solve_ids(pec_ids)
        return job

    @staticmethod
    def _robin_patch(field, dm, plan, ports, robin_bcs, K0, port_vectors):
        """B_p of the reference (``ASM/assembler.py:314-350``) as (distinct CSR slots, summed values) on
        the device: every boundary's 8×8 triangle blocks are added into a per-triangle array in the
        reference's order (ports, then Robin boundaries, each second-order ABC correction after its
        boundary), the nonzero entries are taken in ``generate_csr``'s flat order and summed per slot."""
        dev = dm.device
        mesh = field.mesh
        dpts = dunavant4()
        dp = torch.from_numpy(dpts).to(dev)
        Bflat = torch.zeros((mesh.n_tris, 64), dtype=torch.complex128, device=dev)

        def add(tid, blocks):
            t = torch.from_numpy(np.ascontiguousarray(tid, dtype=np.int64)).to(dev)
            Bflat[t] = Bflat[t] + blocks                       # triangle ids of one boundary are distinct

        for p in ports:
            tid = np.asarray(p.tri_ids, dtype=np.int64)
            tn = mesh.tris[:, tid]
            pts = np.einsum("cvs,vp->cps", mesh.nodes[:, tn], dpts[1:4])
            U = np.asarray(p.get_Uinc(pts[0].ravel(), pts[1].ravel(), pts[2].ravel(), K0), dtype=np.complex128)
            U = torch.from_numpy(np.ascontiguousarray(U.reshape(3, dpts.shape[1], len(tid)))).to(dev)
            blocks, bvec = tri_robin_device(dm, torch.from_numpy(np.ascontiguousarray(tn)).to(dev), p.get_gamma(K0),
                                            U, dp)
            add(tid, blocks)
            bv = bvec.cpu().numpy()
            np.add.at(port_vectors[p.port_number], field.tri_to_field[:, tid].T.ravel(), bv.ravel())
        for bc in robin_bcs:
            tid = np.asarray(bc.tri_ids, dtype=np.int64)
            tn = torch.from_numpy(np.ascontiguousarray(mesh.tris[:, tid])).to(dev)
            add(tid, tri_robin_device(dm, tn, bc.get_gamma(K0))[0])
            if getattr(bc, "order", 1) == 2:                  # second-order ABC correction (:342-347)
                add(tid, tri_abc2_device(dm, tn, bc.get_gamma2(K0)))
        Handle.get(dev).raise_on_device_status("assemble_freq_matrix robin")
        flat = Bflat.reshape(-1)
        ids = torch.nonzero((flat.real != 0) | (flat.imag != 0), as_tuple=False).reshape(-1)
        t2f = torch.from_numpy(np.ascontiguousarray(field.tri_to_field)).to(dev)      # (8, n_tris)
        tri, loc = ids // 64, ids % 64
        rows = t2f[loc // 8, tri]
        cols = t2f[loc % 8, tri]
        slot = plan.find_slots(rows, cols)
        sl = slot.cpu().numpy()
        if (sl < 0).any():
            raise RuntimeError("assemble_freq_matrix: a boundary DOF pair lies outside the tet pattern")
        us, seg, idx = _seg_from_keys(sl)
        vals = gather_sum(torch.from_numpy(seg).to(dev), torch.from_numpy(idx).to(dev), flat[ids].contiguous())
        return torch.from_numpy(us.astype(np.int32)).to(dev), vals


def freq_matrix_device(plan, E: torch.Tensor, B: torch.Tensor, k0sq: float, patch_slot: torch.Tensor | None = None,
                       patch_vals: torch.Tensor | None = None) -> csr_matrix:
    """K = E − B·k0² (+ B_p on distinct slots) formed on the device, exact zeros dropped as SciPy's sparse
    arithmetic drops them, downloaded as a SciPy CSR (int32 indices, sorted rows)."""
    dev = E.device
    h = Handle.get(dev)
    nnz, n = plan.nnz, plan.n_field
    Kf = torch.empty(nnz, dtype=torch.complex128, device=dev)
    npatch = 0 if patch_slot is None else patch_slot.numel()
    check(lib().emfem_sweep_combine(h.h, nnz, ptr(E), ptr(B), float(k0sq), npatch, ptr(patch_slot) if npatch else None,
                                    ptr(patch_vals) if npatch else None, 1.0, 0.0, ptr(Kf)), "emfem_sweep_combine")
    sz = ctypes.c_size_t()
    check(lib().emfem_csr_drop_zeros_workspace(n, ctypes.byref(sz)), "emfem_csr_drop_zeros_workspace")
    ws = torch.empty(sz.value, dtype=torch.uint8, device=dev)
    indptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
    kept = ctypes.c_int64()
    check(lib().emfem_csr_count_nonzero(h.h, n, ptr(plan.indptr), ptr(Kf), ptr(indptr), ptr(ws), ws.numel(),
                                        ctypes.byref(kept)), "emfem_csr_count_nonzero")
    indices = torch.empty(max(kept.value, 1), dtype=torch.int32, device=dev)
    vals = torch.empty(max(kept.value, 1), dtype=torch.complex128, device=dev)
    check(lib().emfem_csr_compact_nonzero(h.h, n, ptr(plan.indptr), ptr(plan.indices), ptr(Kf), ptr(indptr),
                                          ptr(indices), ptr(vals)), "emfem_csr_compact_nonzero")
    h.raise_on_device_status("freq_matrix_device")
    K = csr_matrix((vals[:kept.value].cpu().numpy(), indices[:kept.value].cpu().numpy(), indptr.cpu().numpy()),
                   shape=(n, n))
    K.has_sorted_indices = True
    return K
