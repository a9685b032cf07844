"""CPU oracle for the second-order absorbing-boundary correction — TEST INFRASTRUCTURE ONLY.

A numpy restatement of ``abc_order_2_matrix`` (``src/emerge/_emerge/physics/microwave/assembly/
robin_abc_order2.py:192-373``): per boundary triangle, in its own plane frame (x along the first
edge, z the normal), the 8×8 block cf · L_i L_j · (∫ curl_t N_i curl_t N_j − ∫ div_t N_i div_t N_j) · |A|
with the reference's closed-form tangential curl/divergence polynomials (``:69-150``), barycentric
coefficients (``:157-183``) and its 6-point rule with 8-digit weights and points (``:190-193``).
Pinned against the reference's own output (``tests/golden/abc2.npz``).
"""
from __future__ import annotations

import numpy as np

DPTS = np.array([[0.22338159, 0.22338159, 0.22338159, 0.10995174, 0.10995174, 0.10995174],
                 [0.10810302, 0.44594849, 0.44594849, 0.81684757, 0.09157621, 0.09157621],
                 [0.44594849, 0.44594849, 0.10810302, 0.09157621, 0.09157621, 0.81684757],
                 [0.44594849, 0.10810302, 0.44594849, 0.09157621, 0.81684757, 0.09157621]])
EDGE_MAP = ((0, 1), (1, 2), (0, 2))        # tri_to_edge order (i1,i2),(i2,i3),(i1,i3) of a sorted triangle


def _curl_e1(c, x, y, i, j):
    a1, b1, c1 = c[:, i]; a2, b2, c2 = c[:, j]
    return -3*a1*b1*c2 + 3*a1*b2*c1 - 3*b1**2*c2*x + 3*b1*b2*c1*x - 3*b1*c1*c2*y + 3*b2*c1**2*y


def _curl_e2(c, x, y, i, j):
    a1, b1, c1 = c[:, i]; a2, b2, c2 = c[:, j]
    return -3*a2*b1*c2 + 3*a2*b2*c1 - 3*b1*b2*c2*x - 3*b1*c2**2*y + 3*b2**2*c1*x + 3*b2*c1*c2*y


def _div_e1(c, x, y, i, j):
    a1, b1, c1 = c[:, i]; a2, b2, c2 = c[:, j]
    L1, L2 = a1 + b1*x + c1*y, a2 + b2*x + c2*y
    return b1*(b1*L2 - b2*L1) + c1*(c1*L2 - c2*L1)


def _div_e2(c, x, y, i, j):
    a1, b1, c1 = c[:, i]; a2, b2, c2 = c[:, j]
    L1, L2 = a1 + b1*x + c1*y, a2 + b2*x + c2*y
    return b2*(b1*L2 - b2*L1) + c2*(c1*L2 - c2*L1)


def _face(c, x, y):
    (a1, a2, a3), (b1, b2, b3), (c1, c2, c3) = c
    L1, L2, L3 = a1 + b1*x + c1*y, a2 + b2*x + c2*y, a3 + b3*x + c3*y
    fc1 = -b2*(c1*L3 - c3*L1) + c2*(b1*L3 - b3*L1) + 2*(b1*c3 - b3*c1)*L2
    fc2 = b3*(c1*L2 - c2*L1) - c3*(b1*L2 - b2*L1) - 2*(b1*c2 - b2*c1)*L3
    fd1 = -b2*(b1*L3 - b3*L1) - c2*(c1*L3 - c3*L1)
    fd2 = b3*(b1*L2 - b2*L1) + c3*(c1*L2 - c2*L1)
    return fc1, fc2, fd1, fd2


def tri_block(v: np.ndarray, cf: complex) -> np.ndarray:
    """8×8 correction block of one triangle with vertices v (3, 3) in sorted-node order."""
    o = v[:, 0]
    e1, e2 = v[:, 1] - o, v[:, 2] - o
    z = np.cross(e1, e2); z = z / np.sqrt(z @ z)
    xh = e1 / np.sqrt(e1 @ e1)
    yh = np.cross(z, xh); yh = yh / np.sqrt(yh @ yh)
    loc = np.stack([xh, yh, z]) @ (v - o[:, None])
    xp, yp = loc[0], loc[1]
    D = np.sqrt((xp[:, None] - xp[None]) ** 2 + (yp[:, None] - yp[None]) ** 2)
    W = DPTS[0]
    x = xp[0] * DPTS[1] + xp[1] * DPTS[2] + xp[2] * DPTS[3]
    y = yp[0] * DPTS[1] + yp[1] * DPTS[2] + yp[2] * DPTS[3]
    (x1, x2, x3), (y1, y2, y3) = xp, yp
    a = np.array([x2*y3 - y2*x3, x3*y1 - y3*x1, x1*y2 - y1*x2])
    b = np.array([y2 - y3, y3 - y1, y1 - y2])
    c = np.array([x3 - x2, x1 - x3, x2 - x1])
    sA = 0.5 * ((x1 - x3) * (y2 - y1) - (x1 - x2) * (y3 - y1))
    A = abs(sA)
    s = np.sign(sA)
    bc = np.stack([a * s, b * s, c * s]) / (2 * A)
    Lg = np.ones((8, 8))
    Lg[3, :] *= D[0, 2]; Lg[7, :] *= D[0, 1]; Lg[:, 3] *= D[0, 2]; Lg[:, 7] *= D[0, 1]
    ce = [(_curl_e1(bc, x, y, i, j), _curl_e2(bc, x, y, i, j)) for i, j in EDGE_MAP]
    de = [(_div_e1(bc, x, y, i, j), _div_e2(bc, x, y, i, j)) for i, j in EDGE_MAP]
    for k, (i, j) in enumerate(EDGE_MAP):
        Le = D[i, j]
        Lg[k, :] *= Le; Lg[k + 4, :] *= Le; Lg[:, k] *= Le; Lg[:, k + 4] *= Le
    fc1, fc2, fd1, fd2 = _face(bc, x, y)
    curl = [ce[0][0], ce[1][0], ce[2][0], fc1, ce[0][1], ce[1][1], ce[2][1], fc2]
    div = [de[0][0], de[1][0], de[2][0], fd1, de[0][1], de[1][1], de[2][1], fd2]
    Cm = np.array([[np.sum(p * q * W) for q in curl] for p in curl])
    Dm = np.array([[np.sum(p * q * W) for q in div] for p in div])
    return cf * Lg * (Cm - Dm) * A


def abc_order_2_matrix(field, tri_ids, cf: complex) -> np.ndarray:
    """The reference's flat (N_f·64,) accumulation array with the listed triangles filled."""
    m = field.mesh
    out = np.zeros(m.n_tris * 64, dtype=np.complex128)
    for t in np.asarray(tri_ids, dtype=np.int64):
        out[64 * t:64 * t + 64] += tri_block(m.nodes[:, m.tris[:, t]], cf).ravel()
    return out
