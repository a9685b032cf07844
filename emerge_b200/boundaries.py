"""Robin-type boundaries without excitation: their γ(k0), in the reference's formulas.

Every Robin boundary enters the system as γ(k0) · R̂ with R̂ the triangle matrix of
``assemble_robin_bc`` assembled once with γ = 1 (``ASM/assembler.py:314-350``: the same tri kernel,
only γ differs), so the frequency sweep treats them as extra non-excited "ports".

* :class:`AbsorbingBoundary` — ``MW/microwave_bc.py:282-346``: γ = j k0 (order 1), or j k0 c0 with the
  order-2 coefficient table (the reference's default, ``order=2``, type B) plus the tangential
  correction matrix ``abc_order_2_matrix`` scaled by j c2 / k0 (``ASM/assembler.py:342-347``,
  ``ASM/robin_abc_order2.py:192-373``; device kernel ``emfem_ned2_tri_abc2``).
* :class:`SurfaceImpedance` — ``MW/microwave_bc.py:1243-1343``: γ = j k0 Z0 / Z_s with the skin-depth
  surface impedance of a conductor σ, optional finite thickness (coth) and Hammerstad–Jensen roughness,
  or a user impedance function Z_s(f).

``ASM/`` = ``src/emerge/_emerge/physics/microwave/assembly/``; ``MW/`` = ``src/emerge/_emerge/physics/microwave/``.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable

import numpy as np

from .constants import C0, EPS0, MU0, Z0

__all__ = ["AbsorbingBoundary", "SurfaceImpedance"]

# (c0, c2) of the second-order ABC variants A..E (MW/microwave_bc.py:314-319)
ABC_O2_COEFFS = {"A": (1.0, -0.5), "B": (1.00023, -0.51555), "C": (1.03084, -0.73631),
                 "D": (1.06103, -0.84883), "E": (1.12500, -1.00000)}


@dataclass
class AbsorbingBoundary:
    tri_ids: np.ndarray
    order: int = 2
    abctype: str = "B"

    def __post_init__(self):
        if self.order not in (1, 2):
            raise ValueError("AbsorbingBoundary: order must be 1 or 2")
        if self.abctype not in ABC_O2_COEFFS:
            raise ValueError("AbsorbingBoundary: abctype must be one of A-E")
        self.tri_ids = np.asarray(self.tri_ids, dtype=np.int64)

    def get_gamma2(self, k0: float) -> complex:
        """Coefficient of the second-order correction matrix, j c2 / k0 (0 for order 1)."""
        return 1j * ABC_O2_COEFFS[self.abctype][1] / k0 if self.order == 2 else 0.0

    def get_beta(self, k0: float) -> float:
        return k0

    def get_gamma(self, k0: float) -> complex:
        if self.order == 1:
            return 1j * k0
        return 1j * k0 * ABC_O2_COEFFS[self.abctype][0]


@dataclass
class SurfaceImpedance:
    tri_ids: np.ndarray
    sigma: float = 0.0
    mur: complex = 1.0
    epsr: complex = 1.0
    thickness: float | None = None
    roughness: float = 0.0
    impedance_function: Callable | None = None

    def __post_init__(self):
        self.tri_ids = np.asarray(self.tri_ids, dtype=np.int64)
        if self.impedance_function is None and not self.sigma > 0:
            raise ValueError("SurfaceImpedance: give a conductivity sigma > 0 or an impedance_function")

    def get_beta(self, k0: float) -> float:
        return k0

    def surface_impedance(self, k0: float) -> complex:
        """Z_s(f): skin-depth impedance (1 + j) ρ / δ with the lossy-dielectric skin depth, times
        coth(γ_m t) for a finite layer and the Hammerstad–Jensen roughness factor."""
        w0 = k0 * C0
        if self.impedance_function is not None:
            return complex(self.impedance_function(w0 / (2 * np.pi)))
        eps = EPS0 * self.epsr
        mu = MU0 * self.mur
        rho = 1.0 / self.sigma
        d_skin = (2 * rho / (w0 * mu) * ((1 + (w0 * eps * rho) ** 2) ** 0.5 + rho * w0 * eps)) ** 0.5
        R = (1 + 1j) * rho / d_skin
        if self.thickness is not None:
            eps_c = eps - 1j * self.sigma / w0
            gamma_m = 1j * w0 * np.sqrt(mu * eps_c)
            R = R / np.tanh(gamma_m * self.thickness)
        if self.roughness > 0.0:
            R = R * (1 + 2 / np.pi * np.arctan(1.4 * (self.roughness / d_skin) ** 2))
        return complex(R)

    def get_gamma(self, k0: float) -> complex:
        return 1j * k0 * Z0 / self.surface_impedance(k0)
