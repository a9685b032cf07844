"""S-parameter oracle — TEST INFRASTRUCTURE ONLY (tests call it as the checker).

A numpy restatement of the reference's port-face field interpolation (``ned2_tet_interp``,
``src/emerge/_emerge/elements/ned2_interp.py:142-300``) and overlap integrals (``sparam_field_power``
/ ``sparam_mode_power``, ``src/emerge/_emerge/physics/microwave/sparam.py:71-138``; ``surface_integral``,
``src/emerge/_emerge/mth/integrals.py:60-100``), evaluated in the tet that owns each port triangle
(the only tet containing the triangle's interior quadrature points).  Pinned against the reference's
raw S-matrix in ``tests/test_oracle_golden.py``."""
from __future__ import annotations

import numpy as np


def _tet_coefficients(xs, ys, zs):
    """a, b, c, d (4, n) and V (n) from vertex coordinates (4, n) (``ned2_interp.py:59-77``)."""
    x1, x2, x3, x4 = xs
    y1, y2, y3, y4 = ys
    z1, z2, z3, z4 = zs
    u = np.stack([x2 - x1, y2 - y1, z2 - z1])
    v = np.stack([x3 - x1, y3 - y1, z3 - z1])
    w = np.stack([x4 - x1, y4 - y1, z4 - z1])
    V = np.abs(np.einsum("in,in->n", u, np.cross(v, w, axis=0))) / 6
    a = np.stack([x2*y3*z4 - x2*y4*z3 - x3*y2*z4 + x3*y4*z2 + x4*y2*z3 - x4*y3*z2,
                  -x1*y3*z4 + x1*y4*z3 + x3*y1*z4 - x3*y4*z1 - x4*y1*z3 + x4*y3*z1,
                  x1*y2*z4 - x1*y4*z2 - x2*y1*z4 + x2*y4*z1 + x4*y1*z2 - x4*y2*z1,
                  -x1*y2*z3 + x1*y3*z2 + x2*y1*z3 - x2*y3*z1 - x3*y1*z2 + x3*y2*z1])
    b = np.stack([-y2*z3 + y2*z4 + y3*z2 - y3*z4 - y4*z2 + y4*z3, y1*z3 - y1*z4 - y3*z1 + y3*z4 + y4*z1 - y4*z3,
                  -y1*z2 + y1*z4 + y2*z1 - y2*z4 - y4*z1 + y4*z2, y1*z2 - y1*z3 - y2*z1 + y2*z3 + y3*z1 - y3*z2])
    c = np.stack([x2*z3 - x2*z4 - x3*z2 + x3*z4 + x4*z2 - x4*z3, -x1*z3 + x1*z4 + x3*z1 - x3*z4 - x4*z1 + x4*z3,
                  x1*z2 - x1*z4 - x2*z1 + x2*z4 + x4*z1 - x4*z2, -x1*z2 + x1*z3 + x2*z1 - x2*z3 - x3*z1 + x3*z2])
    d = np.stack([-x2*y3 + x2*y4 + x3*y2 - x3*y4 - x4*y2 + x4*y3, x1*y3 - x1*y4 - x3*y1 + x3*y4 + x4*y1 - x4*y3,
                  -x1*y2 + x1*y4 + x2*y1 - x2*y4 - x4*y1 + x4*y2, x1*y2 - x1*y3 - x2*y1 + x2*y3 + x3*y1 - x3*y2])
    return a, b, c, d, V


def interp_on_owner(mesh, field, solution, tri_ids, dpts) -> np.ndarray:
    """E (3, npts, n_tri) at the quadrature points of boundary triangles, from their owning tets."""
    tri_ids = np.asarray(tri_ids)
    T = mesh.tri_to_tet[0, tri_ids]
    P = np.einsum("cvs,vp->cps", mesh.nodes[:, mesh.tris[:, tri_ids]], dpts[1:4])
    return interp_in_tets(mesh, field, solution, T, P)


def interp_in_tets(mesh, field, solution, T, P) -> np.ndarray:
    """E (3, npts, n) at points P (3, npts, n), the points of column j inside tet T[j]
    (``ned2_tet_interp``, ``ned2_interp.py:230-295``)."""
    T = np.asarray(T)
    tv = mesh.tets[:, T]
    xs, ys, zs = (mesh.nodes[k][tv] for k in range(3))
    a, b, c, d, V = _tet_coefficients(xs, ys, zs)
    V1 = 216 * V ** 3
    F = a[:, None, :] + b[:, None, :] * P[0] + c[:, None, :] * P[1] + d[:, None, :] * P[2]   # (4, npts, nt)
    rank = np.argsort(np.argsort(tv, axis=0), axis=0)
    nt = len(T)
    dpts = np.zeros((1, P.shape[1]))
    cols = np.arange(nt)
    dofs = solution[field.tet_to_field[:, T]]
    grads = (b, c, d)

    def dist(i, j):
        return np.sqrt((xs[i, cols] - xs[j, cols]) ** 2 + (ys[i, cols] - ys[j, cols]) ** 2 + (zs[i, cols] - zs[j, cols]) ** 2)

    def Fat(i):
        return F[i, :, cols].T                                  # (npts, nt)

    E = np.zeros((3, dpts.shape[1], nt), dtype=np.complex128)
    for e, (p, q) in enumerate(((0, 1), (0, 2), (0, 3), (1, 2), (3, 1), (2, 3))):
        swap = rank[p] > rank[q]
        v1 = np.where(swap, q, p)
        v2 = np.where(swap, p, q)
        L = dist(v1, v2)
        F1, F2 = Fat(v1), Fat(v2)
        wgt = dofs[e] * F1 + dofs[10 + e] * F2
        for k in range(3):
            E[k] += L * wgt * (grads[k][v1, cols] * F2 - grads[k][v2, cols] * F1) / V1
    for f, vv in enumerate(((0, 1, 2), (0, 2, 3), (0, 3, 1), (1, 2, 3))):
        vv = np.array(vv)[:, None].repeat(nt, 1)
        srt = np.take_along_axis(vv, np.argsort(np.take_along_axis(rank, vv, 0), axis=0), 0)
        v1, v2, v3 = srt
        L1, L2 = dist(v1, v3), dist(v1, v2)
        F1, F2, F3 = Fat(v1), Fat(v2), Fat(v3)
        Q1 = dofs[6 + f] * L1 * F2
        Q2 = dofs[16 + f] * L2 * F3
        for k in range(3):
            g = grads[k]
            E[k] += (-Q1 * (g[v1, cols] * F3 - g[v3, cols] * F1) + Q2 * (g[v1, cols] * F2 - g[v2, cols] * F1)) / V1
    return E


def sparams(problem, solutions: dict, k0: float, dpts) -> np.ndarray:
    """Raw S-matrix (n_ports, n_ports) from {active port index: solution (N,)} (``_post_process``,
    ``src/emerge/_emerge/physics/microwave/microwave_3d.py:1110-1247``)."""
    mesh, field = problem.mesh, problem.field
    nports = len(problem.ports)
    S = np.full((nports, nports), np.nan + 0j)
    for p, sol in solutions.items():
        for q, port in enumerate(problem.ports):
            if not hasattr(port, "Zmode"):          # lumped port: voltage lines (microwave_3d.py:1271-1291)
                V = lumped_voltage(problem, port, sol)
                a = port.voltage
                b = V - a if q == p else V
                S[q, p] = (b / a) / np.sqrt(problem.ports[p].power)
                continue
            tid = np.asarray(port.tri_ids)
            E = interp_on_owner(mesh, field, sol, tid, dpts)
            tn = mesh.tris[:, tid]
            P = np.einsum("cvs,vp->cps", mesh.nodes[:, tn], dpts[1:4])
            m = port.port_mode_3d_global(P[0], P[1], P[2], k0)
            Q = 1.0 if q == p else 0.0
            ur = problem.ur[:, :, mesh.tri_to_tet[0, tid]]
            const = 1.0 / ((ur[0, 0] + ur[1, 1] + ur[2, 2]) / 3)
            v = mesh.nodes[:, tn]
            A = np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], axis=0), axis=0) / 2
            Zm = port.Zmode(k0)
            fp = np.sum(const * A * np.einsum("p,cpt->t", dpts[0], (E - Q * m) * np.conj(m))) / (2 * Zm)
            mp = np.sum(const * A * np.einsum("p,cpt->t", dpts[0], m * np.conj(m))) / (2 * Zm)
            S[q, p] = fp / mp / np.sqrt(problem.ports[p].power)
    return S


def simpson_line_weights(npl: int) -> np.ndarray:
    """Per-sample weights of ``gauss3_composite`` (``src/emerge/_emerge/coord.py:24-61``) on equally
    spaced samples: its per-section sum (2/3) a + 2 c with a = y0/2 - y1 + y2/2, c = y1 is
    (y0 + 4 y1 + y2) / 3."""
    w = np.ones(npl)
    w[1:-1:2] = 4.0
    w[2:-1:2] = 2.0
    return w / 3.0


def lumped_voltage(problem, port, solution) -> complex:
    """Lumped-port voltage of one solution: the reference's integration lines
    (``define_lumped_port_integration_points``, ``MW/microwave_3d.py:1432-1470``), each point in the
    last face tet containing it (``ned2_tet_interp``'s search, ``ned2_interp.py:174-211``),
    ``Line.line_integral`` (``coord.py:149-153``), averaged over the lines (``microwave_3d.py:1277-1278``)."""
    mesh, field = problem.mesh, problem.field
    nids = np.unique(mesh.tris[:, np.asarray(port.tri_ids)])
    d = np.asarray(port.direction, float)
    xs, ys, zs = mesh.nodes[0, nids], mesh.nodes[1, nids], mesh.nodes[2, nids]
    dot = xs * d[0] + ys * d[1] + zs * d[2]
    starts = np.argwhere(dot == np.min(dot)).flatten()
    ftets = mesh.face_tets(np.asarray(port.tri_ids))
    volts = []
    for k in starts:
        p0 = np.array([xs[k], ys[k], zs[k]])
        p1 = p0 + d * port.height
        pts = np.stack([np.linspace(p0[i], p1[i], 21) for i in range(3)])
        owner = np.full(21, -1)
        for t in ftets:
            v = mesh.nodes[:, mesh.tets[:, t]]
            B = np.linalg.inv(np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]], axis=1))
            loc = B @ (pts - v[:, :1])
            owner[(loc.sum(0) <= 1.00000001) & (loc >= -1e-6).all(0)] = t
        E = interp_in_tets(mesh, field, solution, owner, pts[:, None, :])[:, 0, :]     # (3, 21)
        dl = pts[:, 1] - pts[:, 0]
        volts.append(np.sum(simpson_line_weights(21) * (E[0] * dl[0] + E[1] * dl[1] + E[2] * dl[2])))
    return sum(volts) / len(volts)
