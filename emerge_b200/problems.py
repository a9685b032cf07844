"""Seeded synthetic workloads with the shapes, sizes and value distributions of the benchmark
configurations (no public dataset is involved; meshes come from :func:`mesh.box_tet_mesh`).

* :func:`waveguide`  — air-filled 22.86×10.16×50 mm guide, TE10 ports at z=0 and z=l, PEC on the
  four side walls (the 6 000-tet small case at 10×5×20).
* :func:`cavity`     — dielectric-loaded 0.1 m cube, 40³ hex grid (384 000 tets) by default: each tet
  takes the diagonal εr = εr'(1−j·tanδ) of the last of 8 seeded axis-aligned blocks containing its
  centroid (air elsewhere), εr' ~ U[1,10], tanδ ~ U[1e-4,1e-2], μr = 1; one TE10 port on z=0 and PEC
  on every other face.  The configuration names no excitation, so this port is a choice.
* :func:`substrate_box` — the precision workload: an 80×60×52 hex grid (1 497 600 tets) box with a
  substrate of εr = 3.5 − 0.007j under air and a PEC strip of width W/10 on the interface.  52/5 is not
  an integer, so the interface sits on grid plane round(nz/5) = 10 (z = 10/52 H); its nodes are jittered
  in x and y only, so the interface and the strip stay planar.  Excitation and walls are choices (the
  configuration names none): the strip runs along y between lumped ports (strip to ground, 50 Ω) on the
  two end faces, the rest of the end faces is a second-order absorbing boundary, and the floor (ground),
  lid and side walls are PEC.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import TetMesh, box_tet_mesh
from .nedelec2 import Nedelec2
from .ports import LumpedPort, PortFrame, RectangularWaveguidePort


@dataclass
class Problem:
    name: str
    mesh: TetMesh
    field: Nedelec2
    er: np.ndarray          # (3, 3, N_t) complex
    ur: np.ndarray          # (3, 3, N_t) complex
    ports: list
    pec_tris: np.ndarray
    freqs: np.ndarray
    dims: tuple
    robin: list = field(default_factory=list)   # non-excited Robin boundaries (boundaries.py)

    @property
    def pec_ids(self) -> np.ndarray:
        return self.field.pec_dofs(self.pec_tris)

    @property
    def solve_ids(self) -> np.ndarray:
        return self.field.solve_ids(self.pec_ids)


def identity_tensors(nt: int) -> np.ndarray:
    t = np.zeros((3, 3, nt), dtype=np.complex128)
    for i in range(3):
        t[i, i] = 1.0
    return t


def waveguide(nx=10, ny=5, nz=20, a=22.86e-3, b=10.16e-3, l=50e-3, seed=0, jitter=0.1,
              freqs=(10e9,), shuffle_local=False) -> Problem:
    nodes, tets = box_tet_mesh(nx, ny, nz, a, b, l, jitter=jitter, seed=seed, shuffle_local=shuffle_local)
    mesh = TetMesh(nodes, tets)
    fld = Nedelec2(mesh)
    nt = mesh.n_tets
    ports = [RectangularWaveguidePort(1, PortFrame((a / 2, b / 2, 0.0)), (a, b), mesh.tris_on_plane(2, 0.0)),
             RectangularWaveguidePort(2, PortFrame((a / 2, b / 2, l)), (a, b), mesh.tris_on_plane(2, l))]
    walls = np.concatenate([mesh.tris_on_plane(0, 0.0), mesh.tris_on_plane(0, a),
                            mesh.tris_on_plane(1, 0.0), mesh.tris_on_plane(1, b)])
    return Problem("waveguide", mesh, fld, identity_tensors(nt), identity_tensors(nt), ports, walls,
                   np.asarray(freqs, dtype=np.float64), (a, b, l))


def cavity(n=40, L=0.1, seed=0, jitter=0.1, nblocks=8, nfreq=101, fmin=2e9, fmax=6e9) -> Problem:
    nodes, tets = box_tet_mesh(n, n, n, L, L, L, jitter=jitter, seed=seed)
    mesh = TetMesh(nodes, tets)
    fld = Nedelec2(mesh)
    nt = mesh.n_tets
    rng = np.random.default_rng(seed + 1000)
    cen = (nodes[:, tets[0]] + nodes[:, tets[1]] + nodes[:, tets[2]] + nodes[:, tets[3]]) / 4
    eps = np.ones(nt, dtype=np.complex128)
    for _ in range(nblocks):
        lo = rng.uniform(0, 0.7 * L, 3)
        hi = lo + rng.uniform(0.15 * L, 0.5 * L, 3)
        epr = rng.uniform(1.0, 10.0)
        tand = rng.uniform(1e-4, 1e-2)
        inside = np.all((cen >= lo[:, None]) & (cen <= hi[:, None]), axis=0)
        eps[inside] = epr * (1 - 1j * tand)
    er = np.zeros((3, 3, nt), dtype=np.complex128)
    for i in range(3):
        er[i, i] = eps
    port_tris = mesh.tris_on_plane(2, 0.0)
    ports = [RectangularWaveguidePort(1, PortFrame((L / 2, L / 2, 0.0)), (L, L), port_tris)]
    walls = np.concatenate([mesh.tris_on_plane(0, 0.0), mesh.tris_on_plane(0, L), mesh.tris_on_plane(1, 0.0),
                            mesh.tris_on_plane(1, L), mesh.tris_on_plane(2, L)])
    return Problem("cavity", mesh, fld, er, identity_tensors(nt), ports, walls,
                   np.linspace(fmin, fmax, nfreq), (L, L, L))


def pec_cavity(nx=8, ny=4, nz=12, a=22.86e-3, b=10.16e-3, d=30e-3, seed=0, jitter=0.1) -> Problem:
    """Air-filled rectangular box with PEC on all six faces and no ports (eigenmode workload)."""
    nodes, tets = box_tet_mesh(nx, ny, nz, a, b, d, jitter=jitter, seed=seed)
    mesh = TetMesh(nodes, tets)
    fld = Nedelec2(mesh)
    nt = mesh.n_tets
    walls = np.concatenate([mesh.tris_on_plane(ax, v) for ax, v in ((0, 0.0), (0, a), (1, 0.0), (1, b),
                                                                      (2, 0.0), (2, d))])
    return Problem("pec_cavity", mesh, fld, identity_tensors(nt), identity_tensors(nt), [], walls,
                   np.zeros(0), (a, b, d))


def substrate_box(nx=80, ny=60, nz=52, W=16e-3, L=12e-3, H=10.4e-3, er_sub=3.5 - 0.007j, seed=0, jitter=0.1,
                  nfreq=51, fmin=1e9, fmax=8e9, abc_order=2) -> Problem:
    """Shielded microstrip section (see the module docstring); the strip runs along y."""
    from .boundaries import AbsorbingBoundary
    nodes, tets = box_tet_mesh(nx, ny, nz, W, L, H, jitter=0.0, seed=seed)
    ki = int(round(nz / 5))
    zi = H * ki / nz
    I = np.arange(nodes.shape[1]) % (nx + 1)
    J = (np.arange(nodes.shape[1]) // (nx + 1)) % (ny + 1)
    K = np.arange(nodes.shape[1]) // ((nx + 1) * (ny + 1))
    interior = (I > 0) & (I < nx) & (J > 0) & (J < ny) & (K > 0) & (K < nz)
    rng = np.random.default_rng(seed)
    h = np.array([W / nx, L / ny, H / nz])
    d = rng.uniform(-1.0, 1.0, (3, int(interior.sum()))) * jitter * h[:, None]
    d[2, K[interior] == ki] = 0.0                      # the interface plane stays flat
    nodes = nodes.copy()
    nodes[:, interior] += d
    mesh = TetMesh(nodes, tets)
    fld = Nedelec2(mesh)
    nt = mesh.n_tets
    cz = nodes[2][tets].mean(axis=0)
    er = identity_tensors(nt)
    for i in range(3):
        er[i, i, cz < zi] = er_sub
    cx = mesh.tri_centers()
    half = W / 20
    iface = mesh.tris_on_plane(2, zi)
    strip = iface[np.abs(cx[0, iface] - W / 2) <= half]
    ports, robin = [], []
    for q, y0 in enumerate((0.0, L)):
        face = mesh.tris_on_plane(1, y0)
        sheet = face[(np.abs(cx[0, face] - W / 2) <= half) & (cx[2, face] <= zi)]
        ports.append(LumpedPort(q + 1, sheet, width=2 * half, height=zi, direction=(0.0, 0.0, 1.0), Z0=50.0))
        robin.append(AbsorbingBoundary(np.setdiff1d(face, sheet), order=abc_order))
    walls = np.concatenate([mesh.tris_on_plane(0, 0.0), mesh.tris_on_plane(0, W), mesh.tris_on_plane(2, 0.0),
                            mesh.tris_on_plane(2, H), strip])
    return Problem("substrate_box", mesh, fld, er, identity_tensors(nt), ports, walls,
                   np.linspace(fmin, fmax, nfreq), (W, L, H), robin)


def with_modal_ports(P: Problem, freq: float, nmodes: int = 1, device=None) -> Problem:
    """The same problem with every wave port replaced by a ``ModalPort`` on the same face and frame,
    its mode found by the face eigen-analysis at ``freq``.  Port-face materials are those of the first
    tet owning each triangle (``modal_analysis``, ``microwave_3d.py:536-540``); the edges of the PEC wall
    triangles are PEC for the mode (``assemble_bma_matrices``, ``assembler.py:168-177``)."""
    import dataclasses
    from .ports import ModalPort
    mesh = P.mesh
    pec_edges = mesh.edges[:, mesh.tri_to_edge[:, np.asarray(P.pec_tris, dtype=np.int64)].ravel()]
    ports = []
    for port in P.ports:
        tid = np.asarray(port.tri_ids, dtype=np.int64)
        owner = mesh.tri_to_tet[0, tid]
        mp = ModalPort(port.port_number, tid, port.frame, power=port.power)
        mp.analyse(mesh, P.er[:, :, owner], P.ur[:, :, owner], freq, nmodes=max(nmodes, 1), pec_edges=pec_edges,
                   device=device)
        ports.append(mp)
    return dataclasses.replace(P, ports=ports)


def batch_family(n_meshes: int = 64, seed: int = 7, nfreq: int = 16, aniso_fraction: float = 0.1) -> list:
    """The batched-meshes workload as sweepable problems: ``n_meshes`` box meshes with seeded grid sizes
    giving 5 000-200 000 tets each (the grid and size recipe of the batched assembly benchmark), per-tet
    eps_r' ~ U[1,12] with tan d ~ U[0,5e-3], diagonal mu_r ~ U[1,2]^3 on a seeded ``aniso_fraction`` of
    the tets.  The configuration names no excitation, so each box is a guide section: TE10 ports on the
    z = 0 and z = l faces and PEC on the four side walls.  The analytic TE10 port assumes a homogeneous
    filling, so the cell layer next to each port face holds the member's mean eps_r' (isotropic, same
    loss) while every other tet keeps its own random tensors.  ``nfreq`` frequencies per member span its
    first-mode band, 1.1 to 1.9 times the TE10 cutoff of the mean filling (below the TE20 cutoff)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_meshes):
        target = rng.uniform(5000, 200000) / 6
        nx = max(2, int(round(target ** (1 / 3) * rng.uniform(0.7, 1.3))))
        ny = max(2, int(round((target / nx) ** 0.5 * rng.uniform(0.8, 1.2))))
        nz = max(3, int(round(target / (nx * ny))))
        a = 0.02 * rng.uniform(0.8, 1.25)
        b, l = a * ny / nx, a * nz / nx
        nodes, tets = box_tet_mesh(nx, ny, nz, a, b, l, jitter=0.1, seed=1000 + i)
        mesh = TetMesh(nodes, tets)
        fld = Nedelec2(mesh)
        nt = mesh.n_tets
        epr = rng.uniform(1, 12, nt)
        tand = rng.uniform(0, 5e-3, nt)
        aniso = rng.random(nt) < aniso_fraction
        mu = np.where(aniso[None, :], rng.uniform(1, 2, (3, nt)), 1.0)
        cz = nodes[2][tets].mean(axis=0)
        feed = (cz < l / nz) | (cz > l - l / nz)
        e_mean = float(epr.mean())
        epr = np.where(feed, e_mean, epr)
        mu = np.where(feed[None, :], 1.0, mu)
        er = np.zeros((3, 3, nt), np.complex128)
        ur = np.zeros((3, 3, nt), np.complex128)
        for c in range(3):
            er[c, c] = epr * (1 - 1j * tand)
            ur[c, c] = mu[c]
        ports = [RectangularWaveguidePort(1, PortFrame((a / 2, b / 2, 0.0)), (a, b), mesh.tris_on_plane(2, 0.0),
                                          er=e_mean),
                 RectangularWaveguidePort(2, PortFrame((a / 2, b / 2, l)), (a, b), mesh.tris_on_plane(2, l),
                                          er=e_mean)]
        walls = np.concatenate([mesh.tris_on_plane(0, 0.0), mesh.tris_on_plane(0, a),
                                mesh.tris_on_plane(1, 0.0), mesh.tris_on_plane(1, b)])
        fc = 299792458.0 / (2 * a * np.sqrt(e_mean))
        out.append(Problem(f"batch_member_{i}", mesh, fld, er, ur, ports, walls,
                           np.linspace(1.1 * fc, 1.9 * fc, nfreq), (a, b, l)))
    return out
