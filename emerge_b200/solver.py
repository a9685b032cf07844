"""Solver plugin with the interface of EMerge's solve layer (``src/emerge/_emerge/solver.py``).

* :class:`SolveReport`, :class:`SimulationError`, :class:`Solver` mirror ``solver.py:92-185``,
  ``:295`` and ``:333-371`` (same attributes, method names and return types);
* :class:`SolverB200Krylov` is a ``Solver`` that runs the batched device Krylov solver of libemfem
  (BiCGStab by default, COCG on request; ``SolverB200COCG`` is the same class under its earlier name).  It plugs
  into the reference through ``Simulation.set_solver(instance)`` (``E/simmodel.py:726-734`` →
  ``SolveRoutine.set_solver`` ``solver.py:1079-1090``), as ``SolverCuDSS`` (``:738-773``) does;
* :class:`SolveRoutine` mirrors ``SolveRoutine.solve`` (``:1241-1326``): PEC elimination by
  submatrix ``A[ids, ids]``, solve, scatter back with zeros on eliminated DOFs.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch
from scipy.sparse import csr_matrix

from ._lib import Handle, check, lib, ptr, ERR_NOT_CONVERGED
from .sweep import METHOD, PRECISION, PRECOND


@dataclass
class SolveReport:
    simtime: float = -1.0
    jobid: int = -1
    ndof: int = -1
    nnz: int = -1
    ndof_solve: int = -1
    nnz_solve: int = -1
    exit_code: int = 0
    solver: str = "None"
    sorter: str = "None"
    precon: str = "None"
    aux: dict = field(default_factory=dict)
    worker_name: str = "Unknown Worker"

    def add(self, **kwargs):
        for k, v in kwargs.items():
            self.aux[k] = str(v)

    @property
    def mdof(self) -> float:
        return (self.ndof ** 2) / ((self.simtime + 1e-6) * 1e6)


class SimulationError(Exception):
    pass


class Preconditioner:
    def __init__(self):
        self.M = None

    def init(self, A, b) -> None:
        raise NotImplementedError("")


class Solver:
    """Generic Ax=b solver (``solver.py:333-371``)."""
    real_only: bool = False
    req_sorter: bool = False
    released_gil: bool = False

    def __init__(self, pre: str = ""):
        self.own_preconditioner = False
        self.initialized = False
        self.pre = pre

    def __str__(self) -> str:
        return f"{self.__class__.__name__}"

    def initialize(self) -> None:
        return None

    def duplicate(self) -> "Solver":
        return self.__class__(self.pre)

    def set_options(self, pivoting_threshold: float | None = None) -> None:
        pass

    def solve(self, A, b, precon, reuse_factorization: bool = False, id: int = -1):
        raise NotImplementedError("This classes Ax=B solver method is not implemented.")

    def reset(self) -> None:
        pass


class SolverB200Krylov(Solver):
    """Device Krylov solver (BiCGStab by default, COCG on request), block Jacobi on DOF pairs (i, i+n/2).

    The reference's K is not complex-symmetric (its face-face mass block is asymmetric,
    ``ASM/curlcurl.py:348-357``), so BiCGStab is the default; ``method="cocg"`` is exact only for
    symmetric operators.

    ``solve(A, b)`` takes the already reduced system (SciPy CSR/CSC, complex) exactly as
    ``SolveRoutine.solve`` hands it to a solver.  ``reuse_factorization=True`` keeps the uploaded
    matrix and preconditioner of the previous call (the reference reuses its LU the same way,
    ``MW/simjob.py:105``).  Non-convergence sets ``SolveReport.exit_code = 1`` and logs the FP64 true
    relative residual in ``aux``; ``raise_on_fail=True`` raises :class:`SimulationError` instead.
    """
    real_only = False
    req_sorter = False
    released_gil = True

    def __init__(self, pre: str = "", tol: float = 1e-10, maxit: int = 50000, precond: str = "block_jacobi",
                 precision: str = "fp64", device=None, raise_on_fail: bool = False, method: str = "bicgstab"):
        super().__init__(pre)
        self.tol, self.maxit, self.precond, self.precision = tol, maxit, precond, precision
        self.method = method
        self.device = device
        self.raise_on_fail = raise_on_fail
        self._cache = None

    def duplicate(self) -> "SolverB200Krylov":
        return SolverB200Krylov(self.pre, self.tol, self.maxit, self.precond, self.precision, self.device,
                              self.raise_on_fail, self.method)

    def reset(self) -> None:
        self._cache = None

    def _upload(self, A):
        dev = torch.device("cuda", torch.cuda.current_device()) if self.device is None else torch.device(self.device)
        A = csr_matrix(A)
        A.sort_indices()
        n = A.shape[0]
        if n % 2:
            raise SimulationError("SolverB200Krylov needs the Nedelec-2 DOF pairing (an even number of DOFs)")
        self._cache = dict(
            dev=dev, n=n, nnz=A.nnz,
            indptr=torch.from_numpy(A.indptr.astype(np.int32)).to(dev),
            indices=torch.from_numpy(A.indices.astype(np.int32)).to(dev),
            vals=torch.from_numpy(A.data.astype(np.complex128)).to(dev),
            mask=torch.ones(n, dtype=torch.uint8, device=dev))

    def solve(self, A, b, precon=None, reuse_factorization: bool = False, id: int = -1):
        if not reuse_factorization or self._cache is None:
            self._upload(A)
        c = self._cache
        dev, n = c["dev"], c["n"]
        B = np.asarray(b, dtype=np.complex128)
        multi = B.ndim == 2
        Bm = B if multi else B[:, None]
        nsys = Bm.shape[1]
        out = np.zeros_like(Bm)
        reports = []
        t0 = time.perf_counter()
        for c0 in range(0, nsys, 64):
            cols = Bm[:, c0:c0 + 64]
            ns = cols.shape[1]
            rhs = torch.from_numpy(np.ascontiguousarray(cols)).to(dev)
            x = torch.zeros_like(rhs)
            prec = PRECISION[self.precision]
            sz = ctypes.c_size_t()
            check(lib().emfem_krylov_workspace_size(n, c["nnz"], ns, prec, ctypes.byref(sz)), "emfem_krylov_workspace_size")
            ws = torch.empty(sz.value, dtype=torch.uint8, device=dev)
            status = (ctypes.c_int * ns)(); iters = (ctypes.c_int * ns)(); relres = (ctypes.c_double * ns)()
            k0 = (ctypes.c_double * ns)(*([0.0] * ns))
            h = Handle.get(dev)
            st = lib().emfem_krylov_solve(h.h, METHOD[self.method], n, c["nnz"], ptr(c["indptr"]), ptr(c["indices"]), ptr(c["vals"]), None,
                                        ns, k0, 0, None, None, None, None, None, 0, None, ptr(c["mask"]),
                                        ptr(rhs), ptr(x), self.tol, self.maxit, PRECOND[self.precond], prec,
                                        ptr(ws), ws.numel(), status, iters, relres, None)
            if st not in (0, ERR_NOT_CONVERGED):
                check(st, "emfem_krylov_solve")
            out[:, c0:c0 + ns] = x.cpu().numpy()
            reports.extend(zip(status[:], iters[:], relres[:]))
        simtime = time.perf_counter() - t0
        ok = all(s == 0 for s, _, _ in reports)
        if not ok and self.raise_on_fail:
            raise SimulationError(f"SolverB200Krylov did not converge: {reports}")
        rep = SolveReport(solver=str(self), exit_code=0 if ok else 1, simtime=simtime, precon=self.precond,
                          aux={"iterations": str([r[1] for r in reports]),
                               "true relative residual": str([f"{r[2]:.3e}" for r in reports]),
                               "precision": self.precision, "tolerance": str(self.tol), "method": self.method})
        return (out if multi else out[:, 0]), rep


# earlier name of the class (it runs BiCGStab unless method="cocg")
SolverB200COCG = SolverB200Krylov


class SolveRoutine:
    """``SolveRoutine.solve`` (``solver.py:1241-1326``) with a pluggable solver (default: the device
    Krylov solver)."""

    def __init__(self, solver: Solver | None = None):
        self.forced_solver = [solver] if solver is not None else []
        self.default = SolverB200Krylov()
        self.pre = ""

    def set_solver(self, *solvers: Solver) -> None:
        for s in solvers:
            self.forced_solver = [s]

    def _get_solver(self, A, b) -> Solver:
        for s in self.forced_solver:
            if isinstance(s, Solver):
                return s
        return self.default

    def solve(self, A, b, solve_ids, reuse: bool = False, id: int = -1):
        solver = self._get_solver(A, b)
        solver.initialize()
        NF = A.shape[0]
        A = A.tocsc()
        Asel = A[np.ix_(solve_ids, solve_ids)]
        bsel = b[solve_ids]
        start = time.time()
        x_solved, report = solver.solve(Asel, bsel, None, reuse_factorization=reuse, id=id)
        simtime = time.time() - start
        solution = np.zeros((NF,), dtype=np.complex128)
        solution[solve_ids] = x_solved
        report.jobid = id
        report.simtime = simtime
        report.nnz = A.nnz
        report.ndof = b.shape[0]
        report.nnz_solve = Asel.nnz
        report.ndof_solve = bsel.shape[0]
        report.worker_name = self.pre
        return solution, report
