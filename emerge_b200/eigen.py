"""Eigenmodes of the Nédélec-2 operator with device inner solves.

Replaces the reference's eigenmode path: ``Assembler.assemble_eig_matrix`` (``ASM/assembler.py:431-600``:
E, B with PEC elimination) solved by shift-invert, ``eigs(A, k, M=B, sigma=k_t², which="LM")``
(``SolverARPACK.eig``, ``src/emerge/_emerge/solver.py:820-833``): the eigenpairs of E x = λ M x nearest
σ = k_t², i.e. the dominant eigenvalues ν = 1/(λ − σ) of OP = (E − σM)⁻¹ M.

Ports and Robin boundaries enter as the reference does (``:512-538``): their matrices, with γ taken at
the compile frequency, are added to B, so M = B + Σ γ_p R_p.  On the device that is the sweep operator
with k0² = σ and per-term coefficients −σ γ_p, and the mass product is the sweep SpMV of B with the
Robin patch at coefficients γ_p.

Method: block shift-invert subspace iteration with Rayleigh–Ritz on the pencil.  Each step applies OP
to a block of m vectors as ONE batched device solve (m systems of E − σM, auxiliary-space
preconditioned BiCGStab), orthonormalises the block, projects E and M onto it and solves the small
m × m pencil; the Ritz vectors sorted by |θ − σ| start the next step.  Eigenvalue i converges like
(|λ_i − σ| / |λ_{m+1} − σ|)^k.  The start block comes from a seeded generator, so the result depends
on nothing but the arguments.

Why not ARPACK's generalized mode, as the reference calls it: given M, SciPy runs ARPACK with
``bmat='G'``, which orthogonalises in the M inner product and is only valid for Hermitian positive
semi-definite M.  With port terms M = B + Σ γ_p R_p is complex and non-Hermitian (and the reference's B
is itself not symmetric), and ARPACK then returns Ritz values that are not eigenvalues of the pencil and
change with k and the start vector.  The Rayleigh–Ritz projection here uses Euclidean orthonormal
bases and a dense generalized eigensolver, valid for any M; for a closed PEC cavity (M = B) it finds
the same eigenpairs as the reference.

``ASM/`` = ``src/emerge/_emerge/physics/microwave/assembly/``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.linalg as sla
import torch

from ._lib import Handle, check, lib, ptr
from .constants import C0

__all__ = ["EigenResult", "eigenmodes"]


@dataclass
class EigenResult:
    k0sq: np.ndarray          # eigenvalues λ = k0², sorted by distance to σ
    freqs: np.ndarray         # resonance frequencies (Hz) of the real part of λ
    modes: np.ndarray         # (N, nmodes) complex, zero on PEC DOFs
    inner_solves: int         # systems solved (m per outer step)
    inner_iters: int
    residual: np.ndarray      # ||E x - λ M x|| / (||E x|| + σ ||M x||) per pair (device operators)
    converged: np.ndarray     # residual <= residual_tol
    outer_steps: int = 0


def eigenmodes(sweep, nmodes: int = 4, target_k0: float = 1.0, tol: float = 1e-10, maxit: int = 40000,
               precond: str = "aux", compile_frequency: float | None = None, residual_tol: float = 1e-6,
               seed: int = 0, block: int | None = None, eig_tol: float = 1e-11, max_outer: int = 60) -> EigenResult:
    """The ``nmodes`` eigenpairs of E x = λ (B + Σ γ_p R_p) x nearest σ = target_k0² on the free DOFs
    of a ``FrequencySweep``; γ_p at ``compile_frequency`` (required when the sweep has ports or Robin
    boundaries, as the reference's assemble_eig_matrix takes one frequency for them).

    ``block`` (a power of two, at most 64; default the smallest one >= max(2 nmodes, nmodes + 8)) vectors
    are iterated; the loop stops when every wanted pair's residual is <= ``eig_tol``, when the residuals
    stall, or after ``max_outer`` steps.  ``tol``/``maxit``/``precond`` configure the inner solves.
    Pairs inside the λ = 0 gradient null space of a closed region (nearer σ than the next physical mode
    when σ is low) are not individual eigenpairs; they come back with ``converged`` False unless their
    residual passes."""
    dev = sweep.device
    if nmodes < 1:
        raise ValueError("eigenmodes: nmodes must be >= 1")
    m = block if block is not None else 1 << (max(2 * nmodes, nmodes + 8) - 1).bit_length()
    if m & (m - 1) or not (nmodes <= m <= 64):
        raise ValueError(f"eigenmodes: block {m} must be a power of two in [nmodes, 64]")
    if sweep.n_ports:
        if compile_frequency is None:
            raise ValueError("eigenmodes: a sweep with ports or Robin boundaries needs compile_frequency")
        g = sweep.gammas([compile_frequency])[0]
    else:
        g = np.zeros(0, dtype=np.complex128)
    N = sweep.n
    free = sweep.mask.to(torch.bool)
    sigma = float(target_k0) ** 2
    h = Handle.get(dev)
    zeros_m = torch.zeros(m, dtype=torch.float64, device=dev)
    gm = np.tile(np.stack([g.real, g.imag], -1).reshape(-1), m) if len(g) else np.zeros(2)
    gam_mass = torch.from_numpy(np.ascontiguousarray(gm)).to(dev)
    gam_shift = np.tile((-sigma * g).reshape(1, -1), (m, 1)) if len(g) else None

    def spmv(vals, x, patch: bool):
        # y = vals·x (+ Σ γ_p R_p x when patch) for the m columns of x, PEC rows/cols eliminated
        y = torch.empty_like(x)
        if patch and sweep.n_ports:
            pr = (sweep.patch_rows.numel(), ptr(sweep.patch_rows), ptr(sweep.patch_rowptr), ptr(sweep.patch_cols),
                  ptr(sweep.patch_vals), ptr(sweep.patch_port), sweep.n_ports)
        else:
            pr = (0, None, None, None, None, None, 0)
        check(lib().emfem_sweep_spmv(h.h, N, ptr(sweep.plan.indptr), ptr(sweep.plan.indices), ptr(vals), None, m,
                                     ptr(zeros_m), *pr, ptr(gam_mass), ptr(sweep.mask), ptr(x), ptr(y)),
              "emfem_sweep_spmv")
        return y

    rng = np.random.default_rng(seed)
    v0 = rng.standard_normal((N, m)) + 1j * rng.standard_normal((N, m))
    V = torch.from_numpy(v0).to(dev) * free[:, None]
    solves = iters = 0
    theta = res = None
    outer = 0
    history: list[float] = []
    for outer in range(1, max_outer + 1):
        b = spmv(sweep.B, V.contiguous(), True)
        sol = sweep.solve_rhs([sigma] * m, b, gammas=gam_shift, tol=tol, maxit=maxit, precond=precond)
        solves += m
        iters += int(sol.iters.sum())
        if (sol.status != 0).any():
            raise RuntimeError(f"eigenmodes: inner solve at sigma={sigma:.6g} did not converge "
                               f"(relres {sol.relres.max():.2e} after {sol.iters.max()} iterations)")
        Q, _ = torch.linalg.qr(sol.x)
        Q = (Q * free[:, None]).contiguous()       # Householder reflections spread rounding onto PEC rows
        EQ = spmv(sweep.E, Q, False)
        MQ = spmv(sweep.B, Q, True)
        Eh = (Q.conj().T @ EQ).cpu().numpy()
        Mh = (Q.conj().T @ MQ).cpu().numpy()
        theta, Y = sla.eig(Eh, Mh)
        order = np.argsort(np.abs(theta - sigma))
        theta, Y = theta[order], Y[:, order]
        Yd = torch.from_numpy(np.ascontiguousarray(Y)).to(dev)
        V = Q @ Yd
        nrm = torch.linalg.vector_norm(V, dim=0)
        V = V / nrm
        EV = (EQ @ Yd) / nrm
        MV = (MQ @ Yd) / nrm
        th = torch.from_numpy(theta).to(dev)
        R = EV - MV * th[None, :]
        res = (torch.linalg.vector_norm(R, dim=0) /
               (torch.linalg.vector_norm(EV, dim=0) + sigma * torch.linalg.vector_norm(MV, dim=0))).cpu().numpy()
        worst = float(res[:nmodes].max())
        history.append(worst)
        if worst <= eig_tol:
            break
        # stop when the wanted residuals have stalled for 5 steps (a pair inside the massively degenerate
        # λ ≈ 0 gradient cluster has no well-defined eigenvector and never reaches eig_tol)
        if len(history) > 8 and worst > 0.5 * min(history[-6:-1]):
            break
    modes = V[:, :nmodes].cpu().numpy()
    vals = theta[:nmodes]
    r = res[:nmodes]
    return EigenResult(vals, np.sqrt(np.abs(vals.real)) * C0 / (2 * np.pi), modes, solves, iters, r,
                       r <= residual_tol, outer)
