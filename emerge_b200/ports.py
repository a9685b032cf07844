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

from .constants import C0, EPS0, MU0, Z0


@dataclass
class PortFrame:
    origin: np.ndarray = field(default_factory=lambda: np.zeros(3))
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

    def in_local_cs(self, xyz: np.ndarray) -> np.ndarray:
        """(3, n) global points -> (3, n) local coordinates."""
        return np.array(self.to_local(*np.asarray(xyz, dtype=np.float64)))

    def in_global_basis(self, v: np.ndarray) -> np.ndarray:
        """(3, n) local vector components -> global basis."""
        return np.array(self.to_global_vec(*v))


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


@dataclass
class ModalPort:
    """Wave port whose mode comes from the 2-D eigen-analysis of its face (``ModalPort``,
    ``src/emerge/_emerge/physics/microwave/microwave_bc.py:469-753``, filled by ``modal_analysis``,
    ``microwave_3d.py:474-650``).  Call :meth:`analyse` once; the sweep then uses it like any mode port:

    * beta(k0) = sqrt(beta_m^2 + k0^2 (1 - (f_m / f)^2)) for TE/TM, beta_m k0 / k0_m for TEM (:716-723);
    * Z_mode: Z0 (TEM), k0 c mu0 / beta (TE), beta / (k0 c eps0) (TM) (``PortBC.Zmode``, :218-230);
    * the port field is norm · q(k0) · polarity · E_mode (:650-660) with q = sqrt(Z_mode / Z0) and
      norm = 1 / sqrt(|P q_m^2|), P the mode's power flux (``compute_avg_power_flux``) and q_m the amplitude
      factor ``modal_analysis`` evaluates right after adding the mode (:648): that of the selected entry of
      the modes added so far, i.e. of the first accepted mode when ``mode_number`` is 0;
    * polarity: +1 for the first mode, sign(Re sum e_i^2) for later ones at the same frequency (``add_mode``
      compares each new mode with the last one stored, which is itself, :692-700);
    * modes sorted by descending beta (``sort_modes``, :613-637, no alignment vectors); the sweep uses entry
      ``mode_number``.

    Voltage-line characteristic impedances of TEM ports (``_find_tem_conductors``, :607-632) are not built.
    """
    port_number: int
    tri_ids: np.ndarray
    frame: PortFrame = field(default_factory=PortFrame)
    power: float = 1.0
    active: bool = False
    mode_number: int = 0
    TEM: bool = False

    def __post_init__(self):
        self.tri_ids = np.asarray(self.tri_ids, dtype=np.int64)
        self.modes = []
        self.field = None
        self._ur = None

    def analyse(self, mesh, er, ur, freq: float, nmodes: int = 6, pec_edges=None, sig=None, direct: bool = True,
                target_kz=None, target_neff=None, device=None) -> "ModalPort":
        """Modes of the face at ``freq``; er, ur (3, 3, n_tri) complex tensors of the port triangles."""
        from . import modal
        modes, fld = modal.modal_analysis(mesh, self.tri_ids, self.frame, er, ur, freq, nmodes, direct, self.TEM,
                                          target_kz, target_neff, sig, pec_edges, device, sort=False)
        added = []
        for i, m in enumerate(modes):
            m.polarity = 1.0 if i == 0 else float(np.sign(np.sum(m.modefield * m.modefield).real))
            added.append(m)
            ref = added[min(len(added) - 1, self.mode_number)]
            P = modal.mode_power(fld.mesh, fld, m.modefield, m.k0, ur, m.beta, device)
            m.power = P
            m.norm_factor = float(np.sqrt(1.0 / abs(P * self._qmode_of(ref, m.k0) ** 2)))
        self.modes = sorted(added, key=lambda m: m.beta.real, reverse=True)
        self.field = fld
        self._ur = np.asarray(ur, dtype=np.complex128)
        return self

    @property
    def mode(self):
        if not self.modes:
            raise ValueError("ModalPort: no modes; call analyse() first")
        return self.modes[min(len(self.modes) - 1, self.mode_number)]

    @property
    def polarization(self) -> float:
        return self.mode.polarity

    def modetype(self, k0: float = 0.0) -> str:
        return "TEM" if self.TEM else self.mode.modetype

    @staticmethod
    def _beta_of(m, TEM: bool, k0: float) -> complex:
        if TEM:
            return m.beta / m.k0 * k0
        f = k0 * C0 / (2 * np.pi)
        return np.sqrt(m.beta ** 2 + k0 ** 2 * (1 - (m.freq / f) ** 2))

    def _qmode_of(self, m, k0: float) -> float:
        mt = "TEM" if self.TEM else m.modetype
        beta = self._beta_of(m, self.TEM, k0)
        if mt == "TEM":
            zm = Z0
        elif mt == "TE":
            zm = k0 * C0 / beta * MU0
        else:
            zm = beta / (k0 * C0 * EPS0)
        return np.sqrt(zm / Z0)

    def get_beta(self, k0: float):
        return self._beta_of(self.mode, self.TEM, k0)

    def get_gamma(self, k0: float) -> complex:
        return 1j * self.get_beta(k0)

    def Zmode(self, k0: float):
        return self._qmode_of(self.mode, k0) ** 2 * Z0

    def qmode(self, k0: float):
        return self._qmode_of(self.mode, k0)

    def amplitude(self) -> float:
        return self.mode.norm_factor

    def shape_global(self, x, y, z) -> np.ndarray:
        """Unit-free mode E (global basis) at per-triangle points (npts, n_tri), column t in triangle t."""
        from . import modal
        pts = np.stack([np.asarray(x, float), np.asarray(y, float), np.asarray(z, float)])
        return modal.mode_fields_global(self.field.mesh, self.field, self.mode.modefield, pts)

    def port_mode_3d_global(self, x, y, z, k0: float) -> np.ndarray:
        return self.amplitude() * self.qmode(k0) * self.polarization * self.shape_global(x, y, z)

    def get_Uinc(self, x, y, z, k0: float) -> np.ndarray:
        return -2j * self.get_beta(k0) * self.port_mode_3d_global(x, y, z, k0)

    def uinc_scale(self, k0: float) -> complex:
        return -2j * self.get_beta(k0) * self.qmode(k0) * self.polarization * self.amplitude()
