"""Eigenmodes of the Nédélec-2 operator with device inner solves.

Replaces the reference's eigenmode path: ``Assembler.assemble_eig_matrix`` (``ASM/assembler.py:431-600``:
E, B with PEC elimination) solved by shift-invert ARPACK, ``eigs(A, k, M=B, sigma=k_t², which="LM")``
(``SolverARPACK.eig``, ``src/emerge/_emerge/solver.py:820-833``).  The reference factorises
A − σB inside SciPy; here ARPACK (SciPy, on the host, as in the reference) is given the inverse as an
operator whose every application is a device BiCGStab solve of (E − σB) y = x, preconditioned by the
auxiliary-space correction (σ plays the role of k0²), and the mass products B x run on the device too.
Ports and Robin boundaries enter as the reference does (``:512-538``): their matrices, with γ taken at
the compile frequency, are added to B, so the problem is E x = λ (B + Σ γ_p R_p) x.  On the device that
is the sweep operator with k0² = σ and per-term coefficients −σ γ_p, and the mass product is the
sweep SpMV of B with the Robin patch at coefficients γ_p.

``ASM/`` = ``src/emerge/_emerge/physics/microwave/assembly/``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch
from scipy.sparse.linalg import LinearOperator, eigs

from ._lib import Handle, check, lib, ptr
from .constants import C0

__all__ = ["EigenResult", "eigenmodes"]


@dataclass
class EigenResult:
    k0sq: np.ndarray          # eigenvalues λ = k0², sorted by distance to σ
    freqs: np.ndarray         # resonance frequencies (Hz) of the real part of λ
    modes: np.ndarray         # (N, nmodes) complex, zero on PEC DOFs
    inner_solves: int
    inner_iters: int
    residual: np.ndarray      # ||E x - λ M x|| / (||E x|| + σ ||M x||) per pair (device operators)
    converged: np.ndarray     # residual <= residual_tol


def eigenmodes(sweep, nmodes: int = 4, target_k0: float = 1.0, tol: float = 1e-10, maxit: int = 40000,
               precond: str = "aux", arpack_tol: float = 0.0, compile_frequency: float | None = None,
               residual_tol: float = 1e-6, seed: int = 0) -> EigenResult:
    """The ``nmodes`` eigenpairs of E x = λ (B + Σ γ_p R_p) x nearest σ = target_k0² on the free DOFs
    of a ``FrequencySweep``; γ_p at ``compile_frequency`` (required when the sweep has ports or Robin
    boundaries, as the reference's assemble_eig_matrix takes one frequency for them)."""
    dev = sweep.device
    if sweep.n_ports:
        if compile_frequency is None:
            raise ValueError("eigenmodes: a sweep with ports or Robin boundaries needs compile_frequency")
        g = sweep.gammas([compile_frequency])[0]
    else:
        g = np.zeros(0, dtype=np.complex128)
    free = torch.nonzero(sweep.mask, as_tuple=False).reshape(-1)
    nf = free.numel()
    N = sweep.n
    sigma = float(target_k0) ** 2
    stats = {"solves": 0, "iters": 0}
    h = Handle.get(dev)
    one = torch.zeros(1, dtype=torch.float64, device=dev)
    gm = np.stack([g.real, g.imag], -1).reshape(-1) if len(g) else np.zeros(2)
    gam_mass = torch.from_numpy(np.ascontiguousarray(gm)).to(dev)
    gam_shift = (-sigma * g).reshape(1, -1)

    def full(xf: np.ndarray) -> torch.Tensor:
        x = torch.zeros((N, 1), dtype=torch.complex128, device=dev)
        x[free, 0] = torch.from_numpy(np.ascontiguousarray(xf, dtype=np.complex128)).to(dev)
        return x

    def mass(xf):
        x = full(xf)
        y = torch.empty_like(x)
        # y = (B + Σ γ_p R_p) x through the sweep SpMV with B as its first operator and no second one
        check(lib().emfem_sweep_spmv(h.h, N, ptr(sweep.plan.indptr), ptr(sweep.plan.indices), ptr(sweep.B), None, 1,
                                     ptr(one), sweep.patch_rows.numel(), ptr(sweep.patch_rows),
                                     ptr(sweep.patch_rowptr), ptr(sweep.patch_cols), ptr(sweep.patch_vals),
                                     ptr(sweep.patch_port), sweep.n_ports, ptr(gam_mass), ptr(sweep.mask),
                                     ptr(x), ptr(y)), "emfem_sweep_spmv")
        return y[free, 0].cpu().numpy()

    def opinv(xf):
        res = sweep.solve_rhs([sigma], full(xf), gammas=gam_shift if len(g) else None, tol=tol, maxit=maxit,
                              precond=precond)
        stats["solves"] += 1
        stats["iters"] += int(res.iters.sum())
        if (res.status != 0).any():
            raise RuntimeError(f"eigenmodes: inner solve at sigma={sigma:.6g} did not converge "
                               f"(relres {res.relres.max():.2e} after {res.iters.max()} iterations)")
        return res.x[free, 0].cpu().numpy()

    def stiff(xf):
        raise RuntimeError("not used in shift-invert mode")

    A = LinearOperator((nf, nf), matvec=stiff, dtype=np.complex128)
    M = LinearOperator((nf, nf), matvec=mass, dtype=np.complex128)
    OPinv = LinearOperator((nf, nf), matvec=opinv, dtype=np.complex128)

    def residuals(vals, vecs):
        # ARPACK with an iterative inverse can return a Ritz pair that is not an eigenpair (a strongly
        # damped mode of an open resonator, or an unresolved near-degenerate pair): judge every pair by
        # its residual with the device operators
        res = np.zeros(len(vals))
        for j in range(len(vals)):
            x = full(vecs[:, j])
            ex = torch.empty_like(x)
            check(lib().emfem_sweep_spmv(h.h, N, ptr(sweep.plan.indptr), ptr(sweep.plan.indices), ptr(sweep.E), None,
                                         1, ptr(one), 0, None, None, None, None, None, 0, ptr(gam_mass),
                                         ptr(sweep.mask), ptr(x), ptr(ex)), "emfem_sweep_spmv")
            exf = ex[free, 0].cpu().numpy()
            mx = mass(vecs[:, j])
            r = exf - vals[j] * mx
            # scaled by ||E x|| + σ ||M x||: meaningful for the λ ≈ 0 gradient modes too (E x ≈ 0)
            res[j] = np.linalg.norm(r) / max(np.linalg.norm(exf) + sigma * np.linalg.norm(mx), 1e-300)
        return res

    # ARPACK draws the restart vectors it needs after an invariant subspace from a generator whose
    # state persists in the process, so an unresolved cluster can depend on earlier calls: when a pair
    # fails the residual test, the search is repeated from other seeded start vectors and the attempt
    # with the most converged pairs (then the smallest residual of the nearest pair) is kept
    best = None
    for attempt in range(3):
        v0 = np.random.default_rng(seed + attempt).standard_normal(nf) + 0j      # reproducible start
        vals, vecs = eigs(A, k=nmodes, M=M, sigma=sigma, which="LM", OPinv=OPinv, tol=arpack_tol, v0=v0)
        order = np.argsort(np.abs(vals - sigma))
        vals, vecs = vals[order], vecs[:, order]
        res = residuals(vals, vecs)
        key = (int((res <= residual_tol).sum()), -res[0])
        if best is None or key > best[0]:
            best = (key, vals, vecs, res)
        if (res <= residual_tol).all():
            break
    _, vals, vecs, res = best
    modes = np.zeros((N, nmodes), dtype=np.complex128)
    modes[free.cpu().numpy()] = vecs
    return EigenResult(vals, np.sqrt(np.abs(vals.real)) * C0 / (2 * np.pi), modes, stats["solves"], stats["iters"],
                       res, res <= residual_tol)
