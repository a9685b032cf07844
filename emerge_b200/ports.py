"""Rectangular-waveguide wave port (the port type the sweep configurations use).

Restates ``RectangularWaveguide`` (``src/emerge/_emerge/physics/microwave/microwave_bc.py:755-895``)
and the ``PortBC`` helpers it inherits (``microwave_bc.py:175-280``):

* β = √(εr·k0² − (mπ/w)² − (nπ/h)²), γ = jβ (``:846-862``);
* TE mode field in the port's local frame: E_x' = p·A·sin(mπx'/w)·sin(nπy'/h),
  E_y' = p·A·cos(mπx'/w)·cos(nπy'/h), E_z' = 0, scaled by q = √(Z_mode/Z0) (``:867-883``) with
  A = √(4·P·Z0/(w·h)) (``:839-843``) and Z_mode = k0·c·μ0/β for TE (``:222-230``);
* U_inc = −2jβ·E_mode in global coordinates (``:864-865``).

The port frame is a ``CoordinateSystem``-like (origin, x-, y-, z-axis) with local coordinates
``x' = B⁻¹ (x − origin)`` and vectors mapped back by the axis columns (``cs.py:459-500``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .constants import C0, MU0, Z0


@dataclass
class PortFrame:
    origin: np.ndarray
    xax: np.ndarray = field(default_factory=lambda: np.array([1.0, 0.0, 0.0]))
    yax: np.ndarray = field(default_factory=lambda: np.array([0.0, 1.0, 0.0]))
    zax: np.ndarray = field(default_factory=lambda: np.array([0.0, 0.0, 1.0]))

    def __post_init__(self):
        self.origin = np.asarray(self.origin, dtype=np.float64)
        self.xax = np.asarray(self.xax, float) / np.linalg.norm(self.xax)
        self.yax = np.asarray(self.yax, float) / np.linalg.norm(self.yax)
        self.zax = np.asarray(self.zax, float) / np.linalg.norm(self.zax)
        self.basis = np.array([self.xax, self.yax, self.zax]).T
        self.basis_inv = np.linalg.pinv(self.basis)

    def to_local(self, x, y, z):
        B = self.basis_inv
        xg, yg, zg = x - self.origin[0], y - self.origin[1], z - self.origin[2]
        return (B[0, 0] * xg + B[0, 1] * yg + B[0, 2] * zg,
                B[1, 0] * xg + B[1, 1] * yg + B[1, 2] * zg,
                B[2, 0] * xg + B[2, 1] * yg + B[2, 2] * zg)

    def to_global_vec(self, ex, ey, ez):
        X, Y, Zv = self.xax, self.yax, self.zax
        return (X[0] * ex + Y[0] * ey + Zv[0] * ez,
                X[1] * ex + Y[1] * ey + Zv[1] * ez,
                X[2] * ex + Y[2] * ey + Zv[2] * ez)


@dataclass
class RectangularWaveguidePort:
    """TE_mn wave port on a rectangular face of width ``dims[0]`` (local x) and height ``dims[1]``."""
    port_number: int
    frame: PortFrame
    dims: tuple[float, float]
    tri_ids: np.ndarray
    mode: tuple[int, int] = (1, 0)
    er: float = 1.0
    power: float = 1.0
    polarization: float = 1.0
    active: bool = False

    def get_beta(self, k0: float):
        w, h = self.dims
        return np.sqrt(self.er * k0 ** 2 - (np.pi * self.mode[0] / w) ** 2 - (np.pi * self.mode[1] / h) ** 2)

    def get_gamma(self, k0: float) -> complex:
        return 1j * self.get_beta(k0)

    def Zmode(self, k0: float) -> float:
        return k0 * 299792458 / self.get_beta(k0) * MU0

    def qmode(self, k0: float) -> float:
        return np.sqrt(self.Zmode(k0) / Z0)

    def amplitude(self) -> float:
        return np.sqrt(self.power * 4 * Z0 / (self.dims[0] * self.dims[1]))

    def mode_shape_local(self, xl, yl):
        """(E_x', E_y') of the mode without the k0-dependent factor q·p·A."""
        w, h = self.dims
        m, n = self.mode
        ev = np.cos(np.pi * m * xl / w) * np.cos(np.pi * n * yl / h)
        eh = np.sin(np.pi * m * xl / w) * np.sin(np.pi * n * yl / h)
        return eh, ev

    def port_mode_3d_global(self, x, y, z, k0: float) -> np.ndarray:
        xl, yl, _ = self.frame.to_local(x, y, z)
        w, h = self.dims
        m, n = self.mode
        a = self.polarization * self.amplitude()
        ev = a * np.cos(np.pi * m * xl / w) * np.cos(np.pi * n * yl / h)
        eh = a * np.sin(np.pi * m * xl / w) * np.sin(np.pi * n * yl / h)
        q = self.qmode(k0)
        ex, ey, ez = q * eh, q * ev, q * (0 * eh)
        return np.array(self.frame.to_global_vec(ex, ey, ez))

    def get_Uinc(self, x, y, z, k0: float) -> np.ndarray:
        return -2 * 1j * self.get_beta(k0) * self.port_mode_3d_global(x, y, z, k0)

    def uinc_scale(self, k0: float) -> complex:
        """U_inc(k0) = uinc_scale(k0) · (global-basis mode shape): −2jβ·q·p·A."""
        return -2j * self.get_beta(k0) * self.qmode(k0) * self.polarization * self.amplitude()

    def shape_global(self, x, y, z) -> np.ndarray:
        xl, yl, _ = self.frame.to_local(x, y, z)
        eh, ev = self.mode_shape_local(xl, yl)
        return np.array(self.frame.to_global_vec(eh, ev, 0 * eh))


@dataclass
class LumpedPort:
    """Lumped port (``LumpedPort``, ``src/emerge/_emerge/physics/microwave/microwave_bc.py:1018-1162``):
    a sheet of impedance Z_s = Z0_port·width/height on the port triangles, excited by a uniform field
    along ``direction``.  γ = j k0 Z0 / Z_s (``:1117-1126``); U_inc = −2j k0 (V/height)(Z0/Z_s) · direction
    (``:1128-1130``) with V = √(2 P Z0_port) (``:1100-1106``).  Its S-parameters come from voltage line
    integrals (``microwave_3d.py:1271-1291``; ``FrequencySweep.port_voltages``)."""
    port_number: int
    tri_ids: np.ndarray
    width: float
    height: float
    direction: tuple = (0.0, 0.0, 1.0)
    power: float = 1.0
    Z0: float = 50.0
    active: bool = False

    def __post_init__(self):
        d = np.asarray(self.direction, dtype=np.float64)
        self.direction = d / np.linalg.norm(d)
        self.tri_ids = np.asarray(self.tri_ids, dtype=np.int64)

    @property
    def surfZ(self) -> float:
        return self.Z0 * self.width / self.height

    @property
    def voltage(self) -> float:
        return np.sqrt(2 * self.power * self.Z0)

    def get_beta(self, k0: float) -> float:
        return k0

    def get_gamma(self, k0: float) -> complex:
        return 1j * k0 * Z0 / self.surfZ

    def port_mode_3d_global(self, x, y, z, k0: float = 0.0) -> np.ndarray:
        one = np.ones_like(np.asarray(x, dtype=np.float64))
        return np.array([self.direction[0] * one, self.direction[1] * one, self.direction[2] * one])

    def get_Uinc(self, x, y, z, k0: float) -> np.ndarray:
        return self.uinc_scale(k0) * self.port_mode_3d_global(x, y, z, k0)

    def uinc_scale(self, k0: float) -> complex:
        return -1j * 2 * k0 * self.voltage / self.height * (Z0 / self.surfZ)

    def shape_global(self, x, y, z) -> np.ndarray:
        return self.port_mode_3d_global(x, y, z)


def k0_of(f: float) -> float:
    return 2 * np.pi * f / C0
