"""Frequency-domain assembly with the flow of ``Assembler.assemble_freq_matrix``
(``src/emerge/_emerge/physics/microwave/assembly/assembler.py:189-429``) and the ``SimJob`` it
returns (``src/emerge/_emerge/physics/microwave/simjob.py:23-136``).

Material tensors are passed in directly as (3, 3, N_t) εr/μr arrays (the reference derives them
from ``emsutil.Material`` objects with ``er·(1−j·tanδ) − j·σ/(ωε0)``, ``assembler.py:229-240``);
ports are :class:`~emerge_b200.ports.RectangularWaveguidePort` objects; PEC is a list of boundary
triangles.  The tet and Robin kernels run on the GPU (``assembly.py``); the SciPy steps the
reference performs on the results (``E − B·k0²``, ``generate_csr``, ``K + B_p``) are kept as they
are, so the returned ``K`` is the reference's matrix.
"""
from __future__ import annotations

import numpy as np

from .assembly import (abc_order_2_matrix, assemble_robin_bc, assemble_robin_bc_excited, dunavant4,
                       tet_mass_stiffness_matrices)
from .ports import k0_of


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
        self.cached_matrices = None

    def assemble_freq_matrix(self, field, er: np.ndarray, ur: np.ndarray, ports, pec_tris: np.ndarray,
                             frequency: float, cache_matrices: bool = False, device=None, robin_bcs=()) -> SimJob:
        K0 = k0_of(frequency)
        if cache_matrices and self.cached_matrices is not None:
            E, B = self.cached_matrices
        else:
            E, B = tet_mass_stiffness_matrices(field, er, ur, device=device)
            self.cached_matrices = (E, B)
        K = (E - B * (K0 ** 2)).tocsr()
        b = np.zeros(E.shape[0], dtype=np.complex128)
        port_vectors = {p.port_number: np.zeros(E.shape[0], dtype=np.complex128) for p in ports}
        pec_ids = field.pec_dofs(pec_tris) if len(pec_tris) else np.zeros(0, dtype=np.int64)
        if len(ports) or len(robin_bcs):
            dpts = dunavant4()
            Bempty = field.empty_tri_matrix()
            for p in ports:
                Bempty, b_p = assemble_robin_bc_excited(field, Bempty, p.tri_ids,
                                                        lambda x, y, z, p=p: p.get_Uinc(x, y, z, K0),
                                                        p.get_gamma(K0), dpts, device=device)
                port_vectors[p.port_number] += b_p
            # non-excited Robin boundaries (absorbing, surface impedance): ASM/assembler.py:338-339
            for bc in robin_bcs:
                Bempty = assemble_robin_bc(field, Bempty, bc.tri_ids, bc.get_gamma(K0), device=device)
                if getattr(bc, "order", 1) == 2:        # second-order ABC correction (ASM/assembler.py:342-347)
                    Bempty = Bempty + abc_order_2_matrix(field, bc.tri_ids, bc.get_gamma2(K0), device=device)
            K = K + field.generate_csr(Bempty)
        job = SimJob(K, b, K0 * 299792458 / (2 * np.pi), True)
        job.port_vectors = port_vectors
        job.solve_ids = field.solve_ids(pec_ids)
        return job
