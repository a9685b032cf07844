"""Generate the golden fixtures in this folder by running EMerge's own numba code.

Run in a container that has the reference checkout, with ``EMERGE_REFERENCE_SRC`` set to its
``src/emerge`` folder (required); the GPU box never runs this file, it only reads the
``.npz`` files it wrote.  First numba compile takes about a minute.

    python tests/golden/make_golden.py

Fixtures
--------
``element_small.npz``  72-tet box, shuffled local vertex order, general complex 3×3 εr
    (non-symmetric) and μr (half diagonal, half full): ``_matrix_builder`` COO output
    (``ASM/curlcurl.py:419-466``) and the E/B CSR of ``tet_mass_stiffness_matrices`` (``:145-173``).
``robin_small.npz``    the same mesh's z=0 face through ``assemble_robin_bc_excited`` and its z=l face
    through ``assemble_robin_bc`` (``ASM/robinbc.py:445-473``) with a reference ``RectangularWaveguide``
    TE10 port's γ and U_inc (``MW/microwave_bc.py:846-866``).
``config1.npz``        the 6 000-tet air waveguide (10×5×20 hex grid, 22.86×10.16×50 mm, seed 0) at
    10 GHz with TE10 ports at z=0 and z=l and PEC on the four walls: E/B/K CSR checksums and sampled
    slots, port vectors, both SuperLU solutions (``E/solver.py:561-572`` through the
    ``SolveRoutine.solve`` submatrix path ``:1266-1313``) and the raw S-matrix from the reference's
    ``sparam_field_power``/``sparam_mode_power`` (``MW/sparam.py:71-138``).

``mesh_conn.npz``      two meshes (a shuffled-local-order box and a box with randomly permuted node ids
    and tet order, gmsh-style non-contiguous node tags) through the reference's own
    ``Mesh3D._pre_update`` (``src/emerge/_emerge/mesh3d.py:326-497``), fed by a gmsh stand-in that
    serves the nodes and tets and reports no surface/edge entities: edges, tris, tet_to_edge,
    tet_to_tri, tri_to_edge, tri_to_tet and edge_lengths.

``robin_gamma.npz``    γ(k0) of the reference's ``AbsorbingBoundary`` (order 1, and order 2 types A-E:
    ``MW/microwave_bc.py:282-346``) and ``SurfaceImpedance`` (bulk conductor, finite thickness,
    roughness, user impedance function: ``:1243-1343``) over 2-40 GHz, the objects built without their
    geometry (only the attributes ``get_gamma`` reads are set).

``abc2.npz``           the reference's ``abc_order_2_matrix`` (``ASM/robin_abc_order2.py:350-373``) on the
    element_small mesh's z=0 and x=a faces with coefficient 0.3-0.7j: the touched 64-entry blocks.

``bma.npz``            the boundary-mode-analysis (port-mode) matrices of the reference
    (``ASM/generalized_eigen_hb.py:257-458``): (1) ``_matrix_builder`` on 40 jittered 2-D triangles with
    random vertex and edge orientations and general complex εr/μr tensors (the 14×14 A and B blocks);
    (2) the whole chain of ``Assembler.assemble_bma_matrices`` (``ASM/assembler.py:110-187``) on the z=0
    face of a 10×5×2 WR-90 guide: ``SurfaceMesh`` (``mesh3d.py:717-880``), ``NedelecLegrange2``
    (``elements/nedleg2.py:102-166``), E/B CSR, the PEC DOFs of the four walls, and the eigenvalues of the
    dense ``SolverLAPACK`` path (``solver.py:780-810``) at 10 GHz, for an air-filled guide and one half
    filled with εr = 2.2 - 0.01j; for the top mode, its post-processed vector, E and H from
    ``ned2_tri_interp_full`` / ``ned2_tri_interp_curl`` (``elements/ned2_interp.py:616-760``) at the face's
    order-4 points and its power flux ``compute_avg_power_flux`` (``MW/port_functions.py:21-36``).

Fixtures can be generated one at a time: ``python tests/golden/make_golden.py mesh_conn``.

``ASM/`` = ``src/emerge/_emerge/physics/microwave/assembly/``; ``MW/`` = ``src/emerge/_emerge/physics/microwave/``.
"""
from __future__ import annotations

import hashlib
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import reference_import  # noqa: E402
from emerge_b200.mesh import box_tet_mesh, TetMesh  # noqa: E402
from emerge_b200 import constants as K  # noqa: E402

R = reference_import.load()


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def random_tensors(rng, nt, kind):
    """Complex 3×3 tensors (3, 3, N_t)."""
    if kind == "full":
        t = rng.uniform(0.5, 2.0, (3, 3, nt)) + 1j * rng.uniform(-0.3, 0.3, (3, 3, nt))
        for i in range(3):
            t[i, i] += 3.0
        return t
    if kind == "diag":
        t = np.zeros((3, 3, nt), dtype=np.complex128)
        for i in range(3):
            t[i, i] = rng.uniform(1.0, 4.0, nt) - 1j * rng.uniform(0.0, 0.2, nt)
        return t
    raise ValueError(kind)


def make_port(pnum, origin, dims):
    cs = R.cs.CoordinateSystem(R.cs.Axis(np.array([1.0, 0, 0])), R.cs.Axis(np.array([0, 1.0, 0])),
                               R.cs.Axis(np.array([0, 0, 1.0])), np.array(origin, dtype=np.float64))
    return R.bc.RectangularWaveguide(types.SimpleNamespace(tags=[pnum]), pnum, (1, 0), 1.0, cs, dims)


def element_small():
    nodes, tets = box_tet_mesh(2, 2, 3, 1.0e-2, 0.8e-2, 1.3e-2, jitter=0.15, seed=11, shuffle_local=True)
    mesh = TetMesh(nodes, tets)
    fld = R.nedelec2.Nedelec2(mesh)
    rng = np.random.default_rng(5)
    nt = mesh.n_tets
    er = random_tensors(rng, nt, "full")
    ur = random_tensors(rng, nt, "full")
    ur_diag = random_tensors(rng, nt, "diag")
    ur[:, :, ::2] = ur_diag[:, :, ::2]
    dataE, dataB, rows, cols = R.curlcurl._matrix_builder(
        mesh.nodes, mesh.tets, mesh.tris, mesh.edges, mesh.edge_lengths, fld.tet_to_field,
        mesh.tet_to_edge, ur, er)
    E, B = R.curlcurl.tet_mass_stiffness_matrices(fld, er, ur)
    np.savez_compressed(os.path.join(HERE, "element_small.npz"),
                        nodes=mesh.nodes, tets=mesh.tets, er=er, ur=ur,
                        dataE=dataE, dataB=dataB, rows=rows, cols=cols,
                        E_indptr=E.indptr, E_indices=E.indices, E_data=E.data,
                        B_indptr=B.indptr, B_indices=B.indices, B_data=B.data)
    return mesh, fld


def robin_small(mesh, fld):
    a, b, l = 1.0e-2, 0.8e-2, 1.3e-2
    f = 25e9
    k0 = 2 * np.pi * f / K.C0
    p1 = make_port(1, (a / 2, b / 2, 0.0), (a, b))
    p2 = make_port(2, (a / 2, b / 2, l), (a, b))
    t1 = mesh.tris_on_plane(2, 0.0)
    t2 = mesh.tris_on_plane(2, l)
    DPTs = R.optimized.gaus_quad_tri(4)
    Bm = fld.empty_tri_matrix()
    Bm, bvec = R.robinbc.assemble_robin_bc_excited(fld, Bm, t1, lambda x, y, z: p1.get_Uinc(x, y, z, k0),
                                                   p1.get_gamma(k0), DPTs)
    Bm = R.robinbc.assemble_robin_bc(fld, Bm, t2, p2.get_gamma(k0))
    Bp = fld.generate_csr(Bm)
    touched = np.concatenate([t1, t2])
    blocks = Bm.reshape(-1, 64)[touched]
    np.savez_compressed(os.path.join(HERE, "robin_small.npz"), f=f, k0=k0, tris_port1=t1, tris_port2=t2,
                        gamma1=p1.get_gamma(k0), gamma2=p2.get_gamma(k0), DPTs=DPTs,
                        blocks=blocks, touched=touched, bvec=bvec,
                        Bp_indptr=Bp.indptr, Bp_indices=Bp.indices, Bp_data=Bp.data,
                        beta=p1.get_beta(k0), Zmode=p1.Zmode(k0), amp=p1.get_amplitude(k0))


def config1():
    a, b, l = 22.86e-3, 10.16e-3, 50e-3
    f = 10e9
    nodes, tets = box_tet_mesh(10, 5, 20, a, b, l, jitter=0.1, seed=0)
    mesh = TetMesh(nodes, tets)
    fld = R.nedelec2.Nedelec2(mesh)
    nt = mesh.n_tets
    er = np.zeros((3, 3, nt), dtype=np.complex128)
    ur = np.zeros((3, 3, nt), dtype=np.complex128)
    for i in range(3):
        er[i, i] = 1.0
        ur[i, i] = 1.0
    t0 = time.time()
    E, B = R.curlcurl.tet_mass_stiffness_matrices(fld, er, ur)
    t_asm = time.time() - t0
    k0 = 2 * np.pi * f / K.C0
    Kmat = (E - B * (k0 ** 2)).tocsr()
    ports = [make_port(1, (a / 2, b / 2, 0.0), (a, b)), make_port(2, (a / 2, b / 2, l), (a, b))]
    port_tris = [mesh.tris_on_plane(2, 0.0), mesh.tris_on_plane(2, l)]
    DPTs = R.optimized.gaus_quad_tri(4)
    Bm = fld.empty_tri_matrix()
    port_vectors = {}
    for p, tr in zip(ports, port_tris):
        Bm, bp = R.robinbc.assemble_robin_bc_excited(fld, Bm, tr, lambda x, y, z, p=p: p.get_Uinc(x, y, z, k0),
                                                     p.get_gamma(k0), DPTs)
        port_vectors[p.port_number] = bp
    Kmat = Kmat + fld.generate_csr(Bm)
    walls = np.concatenate([mesh.tris_on_plane(0, 0.0), mesh.tris_on_plane(0, a),
                            mesh.tris_on_plane(1, 0.0), mesh.tris_on_plane(1, b)])
    pec_ids = []
    for ii in mesh.tri_to_edge[:, walls].ravel():
        pec_ids.extend(fld.edge_to_field[:, ii])
    for ii in walls:
        pec_ids.extend(fld.tri_to_field[:, ii])
    pec_set = set(int(i) for i in pec_ids)
    solve_ids = np.array([i for i in range(Kmat.shape[0]) if i not in pec_set])

    routine = R.solver.SolveRoutine()
    sols = {}
    t_solve = []
    for pn, pv in port_vectors.items():
        t0 = time.time()
        x, rep = routine.solve(Kmat, pv, solve_ids, reuse=(pn != 1), id=pn)
        t_solve.append(time.time() - t0)
        sols[pn] = x

    # raw S-matrix through the reference's own overlap integrals (_post_process, microwave_3d.py:1110-1247)
    S = np.zeros((2, 2), dtype=np.complex128)
    for ja, act in enumerate(ports):
        act.active = True
        sol = sols[act.port_number]
        for ib, bc in enumerate(ports):
            tets_face = mesh.face_tets(port_tris[ib])
            fieldf = fld.interpolate_Ef(sol, tetids=tets_face)
            tri_vertices = mesh.tris[:, port_tris[ib]]
            const = np.ones(tri_vertices.shape[1], dtype=np.complex128)   # TE: 1/mean(diag ur) = 1 in air
            fp = R.sparam.sparam_field_power(mesh.nodes, tri_vertices, bc, k0, fieldf, const, 4)
            mp = R.sparam.sparam_mode_power(mesh.nodes, tri_vertices, bc, k0, const, 4)
            S[ib, ja] = (fp / mp) / np.sqrt(act.power)
        act.active = False

    rng = np.random.default_rng(123)
    samp = rng.choice(E.nnz, 4000, replace=False)
    np.savez_compressed(
        os.path.join(HERE, "config1.npz"),
        f=f, k0=k0, nodes_sha=sha(mesh.nodes), tets_sha=sha(mesh.tets),
        n_field=fld.n_field, E_nnz=E.nnz, B_nnz=B.nnz, K_nnz=Kmat.nnz,
        E_indptr=E.indptr.astype(np.int64), E_indices_sha=sha(E.indices.astype(np.int32)),
        K_indptr=Kmat.indptr.astype(np.int64), K_indices_sha=sha(Kmat.indices.astype(np.int32)),
        E_fro=np.linalg.norm(E.data), B_fro=np.linalg.norm(B.data), K_fro=np.linalg.norm(Kmat.data),
        samp=samp, E_samp=E.data[samp], B_samp=B.data[samp], K_samp=Kmat.data[samp],
        E_samp_col=E.indices[samp],
        pv1_idx=np.flatnonzero(port_vectors[1]), pv1_val=port_vectors[1][np.flatnonzero(port_vectors[1])],
        pv2_idx=np.flatnonzero(port_vectors[2]), pv2_val=port_vectors[2][np.flatnonzero(port_vectors[2])],
        n_solve=len(solve_ids), solve_ids_sha=sha(solve_ids.astype(np.int64)),
        x1=sols[1], x2=sols[2], S=S,
        t_assemble_s=t_asm, t_superlu_s=np.array(t_solve))
    print(f"config1: nnz={E.nnz} K.nnz={Kmat.nnz} solve={len(solve_ids)} S=\n{S}\n|S|={np.abs(S)}")


def _reference_mesh3d(nodes, tets, tag_stride=3, tag_offset=7):
    """Run Mesh3D._pre_update on (nodes, tets) through a gmsh stand-in (gmsh node tags are
    tag_offset + tag_stride * (i + 1), tet tags 1..N_t; no 1-D/2-D elements or entities)."""
    import importlib
    gm = sys.modules["gmsh"]
    nn = nodes.shape[1]
    node_tags = (np.arange(1, nn + 1, dtype=np.uint64) * tag_stride + tag_offset)
    empty = np.array([], dtype=np.uint64)

    class _MeshNS:
        @staticmethod
        def get_nodes(*args):
            return node_tags, np.ascontiguousarray(nodes.T).ravel(), None

        @staticmethod
        def get_elements(dim, tag=-1):
            if dim == 3:
                return [4], [np.arange(1, tets.shape[1] + 1, dtype=np.uint64)], [node_tags[tets.T.ravel()]]
            return [], [empty], [empty]

    gm.model = types.SimpleNamespace(mesh=_MeshNS, get_entities=lambda dim=-1: [])
    M = importlib.import_module("emerge._emerge.mesh3d").Mesh3D()
    M._pre_update()
    return M


def mesh_conn():
    out = {}
    nodes, tets = box_tet_mesh(4, 3, 3, 1.0e-2, 0.8e-2, 0.9e-2, jitter=0.15, seed=21, shuffle_local=True)
    cases = {"a": (nodes, tets)}
    rng = np.random.default_rng(77)
    nodes, tets = box_tet_mesh(5, 4, 3, 2.0e-2, 1.0e-2, 1.5e-2, jitter=0.1, seed=22, shuffle_local=True)
    perm = rng.permutation(nodes.shape[1])          # new id of old node i = perm[i]
    nodes_p = np.empty_like(nodes)
    nodes_p[:, perm] = nodes
    tets_p = perm[tets][:, rng.permutation(tets.shape[1])]
    cases["b"] = (nodes_p, tets_p)
    for key, (nd, tt) in cases.items():
        M = _reference_mesh3d(nd, tt)
        out[key + "_nodes"] = nd
        out[key + "_tets"] = np.asarray(M.tets, dtype=np.int64)
        for name in ("edges", "tris", "tet_to_edge", "tet_to_tri", "tri_to_edge", "tri_to_tet"):
            out[key + "_" + name] = np.asarray(getattr(M, name), dtype=np.int64)
        out[key + "_edge_lengths"] = np.asarray(M.edge_lengths, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "mesh_conn.npz"), **out)


def abc2():
    import importlib
    d = np.load(os.path.join(HERE, "element_small.npz"))
    mesh = TetMesh(d["nodes"], d["tets"])
    fld = R.nedelec2.Nedelec2(mesh)
    mod = importlib.import_module("emerge._emerge.physics.microwave.assembly.robin_abc_order2")
    tri = np.concatenate([mesh.tris_on_plane(2, 0.0), mesh.tris_on_plane(0, 1.0e-2)])
    cf = 0.3 - 0.7j
    Mat = mod.abc_order_2_matrix(fld, tri, cf)
    np.savez_compressed(os.path.join(HERE, "abc2.npz"), tri_ids=tri, cf=cf, blocks=Mat.reshape(-1, 64)[tri])


def robin_gamma():
    class _Scalar:
        def __init__(self, v):
            self.v = v

        def scalar(self, f):
            return self.v

    class _Mat:
        def __init__(self, er, ur, cond):
            self.er, self.ur, self.cond = _Scalar(er), _Scalar(ur), _Scalar(cond)

    freqs = np.array([2e9, 5.5e9, 10e9, 24e9, 40e9])
    k0s = 2 * np.pi * freqs / K.C0
    out = {"k0": k0s}
    abc = object.__new__(R.bc.AbsorbingBoundary)
    abc.o2coeffs = {'A': (1.0, -0.5), 'B': (1.00023, -0.51555), 'C': (1.03084, -0.73631),
                    'D': (1.06103, -0.84883), 'E': (1.12500, -1.00000)}
    abc.order = 1
    abc.abctype = 'B'
    out["abc1"] = np.array([abc.get_gamma(k) for k in k0s])
    abc.order = 2
    for t in "ABCDE":
        abc.abctype = t
        out["abc2_" + t] = np.array([abc.get_gamma(k) for k in k0s])
    cases = [dict(sigma=5.8e7, thickness=None, sr=0.0, mur=1.0, er=1.0),
             dict(sigma=3.5e7, thickness=2e-6, sr=0.0, mur=1.0, er=1.0),
             dict(sigma=5.8e7, thickness=None, sr=1.2e-6, mur=1.0, er=1.0),
             dict(sigma=1.0e6, thickness=5e-7, sr=3e-7, mur=1.5, er=2.0)]
    for i, c in enumerate(cases):
        si = object.__new__(R.bc.SurfaceImpedance)
        si._Zf = None
        si.sigma = c["sigma"]
        si.thickness = c["thickness"]
        si._sr = c["sr"]
        si._sr_model = 'Hammerstad-Jensen'
        si._material = _Mat(c["er"], c["mur"], c["sigma"])
        out[f"surf{i}"] = np.array([si.get_gamma(k) for k in k0s])
        out[f"surf{i}_params"] = np.array([c["sigma"], -1.0 if c["thickness"] is None else c["thickness"], c["sr"],
                                           c["mur"], c["er"]])
    si = object.__new__(R.bc.SurfaceImpedance)
    si._Zf = lambda f: (0.02 + 1e-12 * f) + 1j * (0.01 + 3e-12 * f)
    out["surf_fn"] = np.array([si.get_gamma(k) for k in k0s])
    # LumpedPort: γ and U_inc at two points (direction (0.6, 0, 0.8), 2 mm x 3 mm, 50 and 75 ohm)
    for i, (zp, pw) in enumerate(((50.0, 1.0), (75.0, 0.5))):
        lp = object.__new__(R.bc.LumpedPort)
        lp.Z0, lp.width, lp.height, lp.power = zp, 2e-3, 3e-3, pw
        lp.Vdirection = R.cs.Axis(np.array([0.6, 0.0, 0.8]))
        out[f"lumped{i}_gamma"] = np.array([lp.get_gamma(k) for k in k0s])
        xs, ys, zs = np.array([1e-3, 2e-3]), np.array([0.5e-3, 0.0]), np.array([0.0, 1e-3])
        out[f"lumped{i}_uinc"] = np.array([lp.get_Uinc(xs, ys, zs, k) for k in k0s])
    import importlib
    coord = importlib.import_module("emerge._emerge.coord")
    yl = np.random.default_rng(9).standard_normal(21) + 1j * np.random.default_rng(10).standard_normal(21)
    out["line_samples"] = yl
    out["line_gauss3"] = coord.gauss3_composite(np.linspace(0.0, 3e-3, 21), yl)
    np.savez_compressed(os.path.join(HERE, "robin_gamma.npz"), **out)


def bma():
    import importlib
    mesh3d = importlib.import_module("emerge._emerge.mesh3d")
    nl2 = importlib.import_module("emerge._emerge.elements.nedleg2")
    ge = importlib.import_module("emerge._emerge.physics.microwave.assembly.generalized_eigen_hb")
    out = {}
    # (1) element blocks on a jittered 2-D patch with shuffled orientations
    rng = np.random.default_rng(21)
    gx, gy = np.meshgrid(np.linspace(0, 3e-3, 6), np.linspace(0, 2e-3, 5), indexing="ij")
    pts = np.stack([gx.ravel(), gy.ravel()])
    pts = pts + rng.uniform(-0.15, 0.15, pts.shape) * 5e-4
    nid = lambda i, j: i * 5 + j
    tris = []
    for i in range(5):
        for j in range(4):
            tris += [[nid(i, j), nid(i + 1, j), nid(i + 1, j + 1)], [nid(i, j), nid(i + 1, j + 1), nid(i, j + 1)]]
    tris = np.array(tris).T
    tris = np.array([rng.permutation(t) for t in tris.T]).T.astype(np.int64)
    ekey = {}
    t2e = np.zeros((3, tris.shape[1]), dtype=np.int64)
    for t in range(tris.shape[1]):
        for k, (p, q) in enumerate(((0, 1), (1, 2), (0, 2))):
            key = tuple(sorted((int(tris[p, t]), int(tris[q, t]))))
            if key not in ekey:
                ekey[key] = len(ekey)
            t2e[k, t] = ekey[key]
    edges = np.zeros((2, len(ekey)), dtype=np.int64)
    for key, e in ekey.items():
        edges[:, e] = key if rng.random() < 0.5 else key[::-1]
    nt, ne, nn = tris.shape[1], edges.shape[1], pts.shape[1]
    t2f = np.zeros((14, nt), dtype=np.int64)
    t2f[:3] = t2e; t2f[3] = np.arange(nt) + ne; t2f[4:7] = t2e + ne + nt; t2f[7] = np.arange(nt) + 2 * ne + nt
    t2f[8:11] = tris + 2 * ne + 2 * nt; t2f[11:14] = t2e + 2 * ne + 2 * nt + nn
    er = (rng.uniform(1, 4, (3, 3, nt)) + 1j * rng.uniform(-0.2, 0.2, (3, 3, nt)))
    ur = (rng.uniform(0.3, 0.6, (3, 3, nt)) + 1j * rng.uniform(-0.1, 0.1, (3, 3, nt)))
    for i in range(3):
        ur[i, i] += 1.5
    half = np.arange(nt) % 2 == 0
    for i in range(3):
        for j in range(3):
            if i != j:
                ur[i, j, half] = 0
    k0 = 2 * np.pi * 30e9 / K.C0
    local = np.concatenate([pts, np.zeros((1, nn))])
    dE, dB, rows, cols = ge._matrix_builder(local, tris, edges, t2f, ur, er, k0)
    out.update(el_nodes=local, el_tris=tris, el_edges=edges, el_t2f=t2f, el_er=er, el_ur=ur, el_k0=k0,
               el_A=dE.reshape(nt, 196), el_B=dB.reshape(nt, 196), el_rows=rows.reshape(nt, 196),
               el_cols=cols.reshape(nt, 196))
    # (2) the port face of a WR-90 guide through the reference's own surface mesh and field classes
    a, b = 22.86e-3, 10.16e-3
    nodes, tets = box_tet_mesh(10, 5, 2, a, b, 5e-3, seed=0)
    m = TetMesh(nodes, tets)
    tri_ids = m.tris_on_plane(2, 0.0)
    orig = types.SimpleNamespace(tris=m.tris, nodes=m.nodes, edges=m.edges)
    sm = mesh3d.SurfaceMesh(orig, tri_ids, (0.0, 0.0, -1.0))
    cs = R.cs.CoordinateSystem(R.cs.Axis(np.array([1.0, 0, 0])), R.cs.Axis(np.array([0, 1.0, 0])),
                               R.cs.Axis(np.array([0, 0, 1.0])), np.array([0.0, 0, 0]))
    f = nl2.NedelecLegrange2(sm, cs)
    # PEC: every wall triangle's edges mapped into the surface mesh (ASM/assembler.py:168-177)
    walls = np.concatenate([m.tris_on_plane(0, 0.0), m.tris_on_plane(0, a), m.tris_on_plane(1, 0.0),
                            m.tris_on_plane(1, b)])
    pec = []
    for ie in m.tri_to_edge[:, walls].ravel():
        i2 = sm.from_source_edge(ie)
        if i2 is not None:
            pec.extend(list(f.edge_to_field[:, i2]))
    pec = set(int(p) for p in pec)
    solve_ids = np.array([i for i in range(f.n_field) if i not in pec], dtype=np.int64)
    freq = 10e9
    k0 = 2 * np.pi * freq / K.C0
    out.update(wg_a=a, wg_b=b, wg_k0=k0, wg_tri_ids=tri_ids, wg_sm_nodes=sm.nodes, wg_sm_tris=sm.tris,
               wg_sm_edges=sm.edges, wg_sm_tri_to_edge=sm.tri_to_edge, wg_n_field=f.n_field,
               wg_tri_to_field=f.tri_to_field, wg_edge_to_field=f.edge_to_field, wg_solve_ids=solve_ids)
    lap = R.solver.SolverLAPACK("golden")
    for tag, fill in (("air", None), ("half", 2.2 - 0.01j)):
        er = np.zeros((3, 3, sm.n_tris), dtype=np.complex128)
        ur = np.zeros_like(er)
        for i in range(3):
            er[i, i] = 1.0; ur[i, i] = 1.0
        if fill is not None:
            cy = sm.nodes[1][sm.tris].mean(axis=0)
            for i in range(3):
                er[i, i, cy < b / 2] = fill
        E, B = ge.generelized_eigenvalue_matrix(f, er, ur, cs._basis, k0)
        Asel = E[np.ix_(solve_ids, solve_ids)]
        Bsel = B[np.ix_(solve_ids, solve_ids)]
        ermean = 1.0 if fill is None else np.mean(np.diagonal(er[:, :, :]).ravel())
        lam, vecs = lap.eig(Asel, Bsel, 6, 0.7 * k0 * ermean, "LM", sign=-1.0)
        out[f"wg_{tag}_er"] = er
        out[f"wg_{tag}_E_data"], out[f"wg_{tag}_B_data"] = E.data, B.data
        out[f"wg_{tag}_indptr"], out[f"wg_{tag}_indices"] = E.indptr, E.indices
        out[f"wg_{tag}_lambda"] = lam
        top = int(np.argmax(np.sqrt(-lam).real))
        out[f"wg_{tag}_mode"] = vecs[:, top]
        # the mode as modal_analysis post-processes it (MW/microwave_3d.py:576-620): full vector,
        # phase-normalised, beta capped; its E and H at the face's order-4 points and its power flux
        em = np.zeros(f.n_field, dtype=np.complex128)
        em[solve_ids] = vecs[:, top]
        em = em * np.exp(-1j * np.angle(em[np.argmax(np.abs(em))]))
        beta = min(k0 * np.sqrt(np.max(er) * np.max(ur)), np.emath.sqrt(-lam[top]))
        dp = R.optimized.gaus_quad_tri(4)
        v = sm.nodes[:, sm.tris]
        pts = np.einsum("cvs,vp->cps", v, dp[1:4]).reshape(3, -1)
        loc = np.array(cs.in_local_cs(pts[0], pts[1], pts[2]))
        interp = importlib.import_module("emerge._emerge.elements.ned2_interp")
        Ei = np.array(interp.ned2_tri_interp_full(loc[:2].copy(), em, sm.tris, f.local_nodes, f.tri_to_field))
        urinv = np.zeros_like(ur)
        for i in range(sm.n_tris):
            urinv[:, :, i] = R.optimized.matinv(ur[:, :, i])
        Hi = np.array(interp.ned2_tri_interp_curl(loc[:2].copy(), em, sm.tris, f.local_nodes, f.tri_to_field,
                                                  urinv, complex(beta)))
        pf = importlib.import_module("emerge._emerge.physics.microwave.port_functions")
        out[f"wg_{tag}_emode"] = em
        out[f"wg_{tag}_beta"] = complex(beta)
        out[f"wg_{tag}_interpE"] = Ei
        out[f"wg_{tag}_interpH"] = Hi
        out[f"wg_{tag}_power"] = complex(pf.compute_avg_power_flux(f, em, k0, ur, beta))
    out["wg_normal"] = sm.normals[:, 0]
    np.savez_compressed(os.path.join(HERE, "bma.npz"), **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["element_small", "config1", "mesh_conn", "robin_gamma", "abc2", "bma"]
    if "element_small" in which:
        m, f = element_small()
        robin_small(m, f)
    if "config1" in which:
        config1()
    if "mesh_conn" in which:
        mesh_conn()
    if "robin_gamma" in which:
        robin_gamma()
    if "abc2" in which:
        abc2()
    if "bma" in which:
        bma()
    for fn in sorted(os.listdir(HERE)):
        if fn.endswith(".npz"):
            print(fn, os.path.getsize(os.path.join(HERE, fn)))
