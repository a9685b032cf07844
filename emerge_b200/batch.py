"""Many uneven meshes assembled in one launch.

The reference assembles one mesh per ``tet_mass_stiffness_matrices`` call (``ASM/curlcurl.py:145-173``).
:class:`MeshBatch` concatenates a list of meshes into one disjoint union: node ids of mesh k are
offset by the node counts of meshes 0..k-1.  It computes the union's connectivity on the device
(:class:`connectivity.DeviceTetMesh`), builds one symbolic plan and assembles E and B of every mesh
with one launch of the fused kernel.

Union ids keep each mesh contiguous.  Unique edges and triangles are sorted lexicographically by node
id, and the offsets increase with k, so mesh k's edges form one contiguous range of the union's edges
and its triangles one range of the union's triangles.  Its DOFs are therefore the four ranges
[edges_k | faces_k | edges_k + H | faces_k + H] (``elements/nedelec2.py:42-58``).  Each row of the
union CSR lists exactly mesh k's columns, in mesh k's own order.  Each value is summed over the same
tets in the same order as a separate assembly.  :meth:`MeshBatch.csr` therefore returns every mesh's
matrices bit for bit equal to assembling that mesh alone.

:class:`BatchSweep` goes one step further: the frequency sweeps of all meshes run as ONE batched Krylov
call (``emfem_krylov_solve_grouped``).  The union CSR is permuted so that every mesh's DOF pairs form one
contiguous range of whole 256-pair blocks (padded with eliminated rows); each mesh is a group of the
same number of systems, and each system keeps its own BiCGStab scalars and convergence test while one
graph-captured iteration serves all of them.

``ASM/`` = ``src/emerge/_emerge/physics/microwave/assembly/``.
"""
from __future__ import annotations

import time
from types import SimpleNamespace

import numpy as np
import torch
from scipy.sparse import csr_matrix

from .assembly import CsrPlan, DeviceMesh
from .connectivity import DeviceTetMesh

__all__ = ["MeshBatch", "BatchSweep", "grouped_layout"]


class MeshBatch:
    def __init__(self, meshes, device=None):
        """meshes: list of (nodes (3, N_n), tets (4, N_t)) in Mesh3D layouts (host or device)."""
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = dev
        nodes, tets, self.node_off, self.tet_off = [], [], [0], [0]
        for nd, tt in meshes:
            nd = torch.as_tensor(np.asarray(nd) if not isinstance(nd, torch.Tensor) else nd).to(dev, torch.float64)
            tt = torch.as_tensor(np.asarray(tt) if not isinstance(tt, torch.Tensor) else tt).to(dev, torch.int64)
            nodes.append(nd)
            tets.append(tt + self.node_off[-1])
            self.node_off.append(self.node_off[-1] + nd.shape[1])
            self.tet_off.append(self.tet_off[-1] + tt.shape[1])
        self.n_meshes = len(meshes)
        self.mesh = DeviceTetMesh(torch.cat(nodes, dim=1), torch.cat(tets, dim=1), dev)
        self.dmesh = DeviceMesh(self.mesh, None, dev)
        self.plan = CsrPlan(self.dmesh)
        # per-mesh entity ranges: edges/tris whose first (smallest) node lies in the mesh's node range
        no = torch.tensor(self.node_off, device=dev)
        self.edge_off = torch.searchsorted(self.mesh.edges[0].contiguous(), no).cpu().numpy()
        self.tri_off = torch.searchsorted(self.mesh.tris[0].contiguous(), no).cpu().numpy()
        self.E = self.B = None

    @property
    def n_tets(self) -> int:
        return self.tet_off[-1]

    def assemble(self, er: torch.Tensor, ur: torch.Tensor):
        """One fused launch for every mesh; er/ur (3, 3, total tets) complex (mesh order)."""
        self.E, self.B = self.plan.assemble(er, ur, self.E, self.B)
        return self.E, self.B

    def dof_ranges(self, k: int) -> list[tuple[int, int]]:
        """Mesh k's DOFs in the union numbering: [edges | faces | edges + H | faces + H]."""
        ne, nf = self.dmesh.n_edges, self.dmesh.n_tris
        H = ne + nf
        e0, e1 = int(self.edge_off[k]), int(self.edge_off[k + 1])
        t0, t1 = int(self.tri_off[k]), int(self.tri_off[k + 1])
        return [(e0, e1), (ne + t0, ne + t1), (H + e0, H + e1), (H + ne + t0, H + ne + t1)]

    def csr(self, k: int, which: str = "E") -> csr_matrix:
        """Mesh k's E or B as a SciPy CSR in its own DOF numbering (host copy)."""
        vals = (self.E if which == "E" else self.B).cpu().numpy()
        indptr, indices = self.plan.host_pattern()
        ranges = self.dof_ranges(k)
        rows = np.concatenate([np.arange(a, b) for a, b in ranges])
        n = len(rows)
        local = np.full(self.plan.n_field, -1, dtype=np.int64)
        local[rows] = np.arange(n)
        starts, ends = indptr[rows], indptr[rows + 1]
        sel = np.concatenate([np.arange(s, e) for s, e in zip(starts, ends)])
        cols = local[indices[sel]]
        if (cols < 0).any():
            raise RuntimeError("MeshBatch: a row couples two meshes (inputs are not disjoint)")
        new_ptr = np.concatenate([[0], np.cumsum(ends - starts)])
        return csr_matrix((vals[sel], cols.astype(np.int32), new_ptr.astype(np.int32)), shape=(n, n))


def grouped_layout(n_edges, n_tris, align: int = 256):
    """Row layout of the grouped multi-mesh system.

    The union of G meshes numbers its DOFs [edges | faces | edges + H | faces + H] over all meshes, with
    mesh g's edges at [eo_g, eo_g + n_edges[g]) and faces at [to_g, to_g + n_tris[g]) (the offsets are
    the running sums).  The grouped layout puts mesh g's DOF pairs (first kind at i, second kind at
    i + h) at [hoff[g], hoff[g] + H_g) with H_g = n_edges[g] + n_tris[g] padded to a multiple of
    ``align``, in mesh g's own order (its edges, then its faces).  Returns (hoff (G + 1,), perm) with
    perm[u] the grouped row of union DOF u."""
    ne_g = np.asarray(n_edges, dtype=np.int64)
    nf_g = np.asarray(n_tris, dtype=np.int64)
    Hg = ne_g + nf_g
    Hp = (Hg + align - 1) // align * align
    hoff = np.concatenate([[0], np.cumsum(Hp)]).astype(np.int64)
    eo = np.concatenate([[0], np.cumsum(ne_g)])
    to = np.concatenate([[0], np.cumsum(nf_g)])
    ne, nf = int(eo[-1]), int(to[-1])
    x = np.arange(ne + nf, dtype=np.int64)
    is_e = x < ne
    g_e = np.searchsorted(eo, x[is_e], side="right") - 1
    g_f = np.searchsorted(to, x[~is_e] - ne, side="right") - 1
    first = np.empty(ne + nf, dtype=np.int64)
    first[is_e] = hoff[g_e] + (x[is_e] - eo[g_e])
    first[~is_e] = hoff[g_f] + ne_g[g_f] + (x[~is_e] - ne - to[g_f])
    return hoff, np.concatenate([first, first + hoff[-1]])


class BatchSweep:
    """Sweeps of several problems (``problems.Problem``: mesh, materials, ports, PEC, Robin boundaries)
    solved together.  Assembly: one fused launch for all meshes (:class:`MeshBatch`).  Solve: one
    batched call per :meth:`solve`, ``nsys`` systems per mesh."""

    PAIR_ALIGN = 256

    def __init__(self, problems, device=None):
        from .sweep import FrequencySweep
        self.problems = list(problems)
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = dev
        self.batch = MeshBatch([(P.mesh.nodes, P.mesh.tets) for P in self.problems], dev)
        er = torch.cat([torch.from_numpy(np.ascontiguousarray(P.er)) for P in self.problems], dim=2).to(dev)
        ur = torch.cat([torch.from_numpy(np.ascontiguousarray(P.ur)) for P in self.problems], dim=2).to(dev)
        E, B = self.batch.assemble(er, ur)                      # one launch for every mesh
        del er, ur
        # grouped layout: mesh g's DOF pairs at [hoff[g], hoff[g] + H_g) of each half, padded to 256
        G = len(self.problems)
        b = self.batch
        ne_g = np.diff(b.edge_off.astype(np.int64))
        nf_g = np.diff(b.tri_off.astype(np.int64))
        if not (np.array_equal(ne_g, [P.mesh.n_edges for P in self.problems])
                and np.array_equal(nf_g, [P.mesh.n_tris for P in self.problems])):
            raise RuntimeError("BatchSweep: the union's entity ranges do not match the meshes")
        self.hoff, perm = grouped_layout(ne_g, nf_g, self.PAIR_ALIGN)
        self.Hg = ne_g + nf_g
        self.h = int(self.hoff[-1])
        self.n = 2 * self.h
        Hp = np.diff(self.hoff)
        self.pair_group = torch.from_numpy(np.repeat(np.arange(G, dtype=np.int32), Hp)).to(dev)
        inv = np.full(self.n, -1, dtype=np.int64)
        inv[perm] = np.arange(perm.size)
        # grouped CSR: rows moved, columns relabelled (their order inside a row is kept)
        indptr_u = b.plan.indptr.to(torch.int64)
        lens_u = indptr_u[1:] - indptr_u[:-1]
        inv_d = torch.from_numpy(inv).to(dev)
        has = inv_d >= 0
        lens = torch.zeros(self.n, dtype=torch.int64, device=dev)
        lens[has] = lens_u[inv_d[has]]
        indptr = torch.zeros(self.n + 1, dtype=torch.int64, device=dev)
        indptr[1:] = torch.cumsum(lens, 0)
        nnz = int(indptr[-1])
        row_of_slot = torch.repeat_interleave(torch.arange(self.n, device=dev), lens)
        start_u = torch.zeros(self.n, dtype=torch.int64, device=dev)
        start_u[has] = indptr_u[:-1][inv_d[has]]
        slot = start_u[row_of_slot] + (torch.arange(nnz, device=dev) - indptr[:-1][row_of_slot])
        perm_d = torch.from_numpy(perm).to(dev)
        self.indices = perm_d[b.plan.indices.to(torch.int64)[slot]].to(torch.int32).contiguous()
        self.indptr = indptr.to(torch.int32).contiguous()
        self.E = E[slot].contiguous()
        self.B = B[slot].contiguous()
        self.nnz = nnz
        self.plan = SimpleNamespace(indptr=self.indptr, indices=self.indices, nnz=nnz)
        # the union-ordered values are not needed again: keep one copy of E and B on the device
        self.batch.E = self.batch.B = None
        del E, B
        self._perm = perm_d
        self._aux = None
        self.network = None
        del slot, row_of_slot, start_u, lens
        # per mesh: Robin / port terms and port vectors (built on each mesh's own numbering), mask
        self.sweeps = []
        mask = torch.zeros(self.n, dtype=torch.uint8, device=dev)
        rows_l, ptr_l, cols_l, port_l, vals_l = [], [], [], [], []
        nrow_off = 0
        nslot_off = 0
        self.n_ports = 0
        for g, P in enumerate(self.problems):
            fs = FrequencySweep.port_terms(P, dev)
            self.sweeps.append(fs)
            loc = self.local_to_grouped(g)
            mask[loc] = fs.mask
            self.n_ports = max(self.n_ports, fs.n_ports)
            if fs.patch_rows.numel():
                rows_l.append(loc[fs.patch_rows.long()].to(torch.int32))
                ptr_l.append((fs.patch_rowptr[:-1] + nslot_off).to(torch.int32))
                cols_l.append(loc[fs.patch_cols.long()].to(torch.int32))
                port_l.append(fs.patch_port)
                vals_l.append(fs.patch_vals)
                nrow_off += fs.patch_rows.numel()
                nslot_off += fs.patch_vals.numel()
        if self.n_ports > 8:
            raise ValueError("at most 8 ports + Robin terms per mesh")
        i32 = dict(dtype=torch.int32, device=dev)
        self.mask = mask
        self.patch_rows = torch.cat(rows_l) if rows_l else torch.zeros(0, **i32)
        self.patch_rowptr = torch.cat(ptr_l + [torch.tensor([nslot_off], **i32)]) if ptr_l else torch.zeros(1, **i32)
        self.patch_cols = torch.cat(cols_l) if cols_l else torch.zeros(0, **i32)
        self.patch_port = torch.cat(port_l) if port_l else torch.zeros(0, **i32)
        self.patch_vals = torch.cat(vals_l) if vals_l else torch.zeros(0, dtype=torch.complex128, device=dev)
        self._ws = None

    def local_to_grouped(self, g: int) -> torch.Tensor:
        """Rows of the grouped system holding mesh g's DOFs, in that mesh's own DOF order."""
        H = int(self.Hg[g])
        d = torch.arange(2 * H, device=self.device)
        return torch.where(d < H, self.hoff[g] + d, self.h + self.hoff[g] + d - H)

    def solve(self, systems, tol: float = 1e-8, maxit: int = 20000, precond: str = "block_jacobi",
              method: str = "bicgstab", precision: str = "fp64"):
        """systems: one list of (frequency, port) per mesh, all of the same length (<= 64).  Returns one
        ``SolveResult`` per mesh, solutions in that mesh's own DOF numbering."""
        import ctypes
        from ._lib import ERR_NOT_CONVERGED, Handle, check, lib, ptr
        from .ports import k0_of
        from .sweep import METHOD, PRECISION, PRECOND, SolveResult
        G = len(self.problems)
        if len(systems) != G or len({len(s) for s in systems}) != 1:
            raise ValueError("give the same number of systems for every mesh")
        nsys = len(systems[0])
        if PRECOND[precond] == 4 and self.network is None:
            raise ValueError("precond='learned' needs a network (BatchSweep.set_network)")
        npt = max(self.n_ports, 1)
        k0 = np.zeros(G * nsys)
        gam = np.zeros((G * nsys, npt), dtype=np.complex128)
        b = torch.zeros((self.n, nsys), dtype=torch.complex128, device=self.device)
        for g, (fs, sl) in enumerate(zip(self.sweeps, systems)):
            loc = self.local_to_grouped(g)
            freqs = [f for f, _ in sl]
            k0[g * nsys:(g + 1) * nsys] = fs.k0sq(freqs)
            if fs.n_ports:
                gam[g * nsys:(g + 1) * nsys, :fs.n_ports] = fs.gammas(freqs)
            if fs.problem.ports:
                b[loc] = fs.rhs(sl)
        ga = np.ascontiguousarray(np.stack([gam.real, gam.imag], axis=-1).reshape(-1))
        sz = ctypes.c_size_t()
        prec = PRECISION[precision]
        check(lib().emfem_krylov_workspace_size_grouped(self.n, self.nnz, nsys, G, prec, ctypes.byref(sz)),
              "emfem_krylov_workspace_size_grouped")
        if self._ws is None or self._ws.numel() < sz.value:
            self._ws = torch.empty(sz.value, dtype=torch.uint8, device=self.device)
        x = torch.zeros_like(b)
        st = (ctypes.c_int * (G * nsys))()
        it = (ctypes.c_int * (G * nsys))()
        rr = (ctypes.c_double * (G * nsys))()
        aux = None
        pc = PRECOND[precond]
        if pc == 4 and not self.network.active():
            pc = PRECOND["aux"]                # zero output weights: the aux Jacobi exactly, no layers to run
        if pc >= 3:
            a = self.aux_space()
            a.reserve(nsys)
            aux = a.handle
        h = Handle.get(self.device)
        t0 = time.perf_counter()
        rc = lib().emfem_krylov_solve_grouped(
            h.h, METHOD[method], self.n, self.nnz, ptr(self.indptr), ptr(self.indices), ptr(self.E), ptr(self.B), G,
            ptr(self.pair_group), nsys, (ctypes.c_double * (G * nsys))(*k0), self.patch_rows.numel(),
            ptr(self.patch_rows), ptr(self.patch_rowptr), ptr(self.patch_cols), ptr(self.patch_vals),
            ptr(self.patch_port), self.n_ports, (ctypes.c_double * len(ga))(*ga), ptr(self.mask), ptr(b), ptr(x),
            tol, maxit, pc, prec, ptr(self._ws), self._ws.numel(), st, it, rr, aux)
        torch.cuda.synchronize(self.device)
        dt = time.perf_counter() - t0
        if rc not in (0, ERR_NOT_CONVERGED):
            check(rc, "emfem_krylov_solve_grouped")
        out = []
        for g, sl in enumerate(systems):
            sel = slice(g * nsys, (g + 1) * nsys)
            out.append(SolveResult(x[self.local_to_grouped(g)].contiguous(), np.array(st[sel]), np.array(it[sel]),
                                   np.array(rr[sel]), list(sl), dt))
        return out

    def aux_space(self):
        """The auxiliary nodal space of all meshes (their disjoint union, built once), moved onto the
        grouped rows, with the grouped operator's diagonals: ``precond="aux"`` for every mesh at once."""
        if self._aux is None:
            from .auxspace import AuxSpace
            Ps = self.problems
            G = len(Ps)
            nn = np.array([P.mesh.n_nodes for P in Ps])
            ne = np.array([P.mesh.n_edges for P in Ps])
            nn_off = np.concatenate([[0], np.cumsum(nn)])
            ne_off = np.concatenate([[0], np.cumsum(ne)])
            union = SimpleNamespace(
                nodes=np.zeros((3, int(nn_off[-1]))),
                edges=np.concatenate([P.mesh.edges + nn_off[g] for g, P in enumerate(Ps)], axis=1),
                tris=np.concatenate([P.mesh.tris + nn_off[g] for g, P in enumerate(Ps)], axis=1),
                tri_to_edge=np.concatenate([P.mesh.tri_to_edge + ne_off[g] for g, P in enumerate(Ps)], axis=1),
                edge_lengths=np.concatenate([P.mesh.edge_lengths for P in Ps]))
            aux = AuxSpace(union, self.device)
            grp = np.concatenate([np.repeat(np.arange(G), nn), np.repeat(np.arange(G), ne)]).astype(np.int32)
            aux.set_rows(self._perm, self.n, torch.from_numpy(grp) if G > 1 else None)
            aux.set_operator(self)
            self._aux = aux
        return self._aux

    def set_network(self, net) -> None:
        """Use this :class:`auxspace.Network` for ``precond="learned"`` on every mesh (its weights are per
        aux-node type, so a network trained on one mesh applies to the union)."""
        self.network = net
        self.aux_space().set_network(net.params if net is not None else None)

    def sparams(self, g: int, res) -> dict:
        """S-parameters of mesh g's solved systems (``FrequencySweep.sparams``)."""
        return self.sweeps[g].sparams(res)


def solve_meshes_partitioned(problems, systems, world_size: int | None = None, rank: int | None = None,
                             **kw) -> list[list[dict]]:
    """Many meshes' sweeps across the ranks of the process group: meshes are dealt by cost (DOFs x systems,
    the work of one batched Krylov iteration over the mesh's systems), each rank solves its meshes in one
    :class:`BatchSweep` call on its own GPU (keyword arguments passed to ``BatchSweep.solve``), and every
    rank gets, per mesh in input order, one dict per system (status, iterations, FP64 relative residual)."""
    from . import distributed
    ws, rk = distributed.world()
    ws = ws if world_size is None else world_size
    rk = rk if rank is None else rank
    items = list(range(len(problems)))
    cost = [float(problems[i].field.n_field) * len(systems[i]) for i in items]
    mine = [i for i, _ in distributed.partition(items, ws, rk, cost)]
    local = []
    if mine:
        res = BatchSweep([problems[i] for i in mine]).solve([systems[i] for i in mine], **kw)
        for i, r in zip(mine, res):
            local.append((i, [{"status": int(r.status[j]), "iters": int(r.iters[j]), "relres": float(r.relres[j])}
                              for j in range(len(systems[i]))]))
    return distributed.gather(local, len(problems))
