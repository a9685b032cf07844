"""Device sparse direct solver (multifrontal LU over a nested-dissection tree) for the sweep systems.

Replaces the reference's direct solve, ``SolverSuperLU.solve`` (``src/emerge/_emerge/solver.py:535-572``:
SuperLU with MMD ordering), reached through ``SolveRoutine.solve`` (``:1241-1326``).

Ordering (host, once per mesh).  Unknowns are grouped by the mesh entity (edge or face) that owns
them, the first- and second-kind DOFs X and X + H of ``elements/nedelec2.py:42-58``.  Two entities
couple exactly when they share a tet, so a set of entities shared by two disjoint tet sets separates
them.  The tets are bisected recursively along the longest axis of their centroids, at the widest gap
between sorted centroids near the median (for a layered mesh that is a plane between two cell
layers); the entities shared by both halves form the separator of that tree node, and the halves
recurse.  Leaves hold at most ``leaf_tets`` tets.  Every tree node owns its entities' free DOFs; its
front is those DOFs followed by its boundary: the DOFs of ancestor entities that share a tet with
an entity of the node's subtree, in elimination order.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["EliminationTree", "nested_dissection", "FrontStructure", "front_structure", "DeviceLU"]


@dataclass
class EliminationTree:
    """Nested-dissection tree in postorder (children before parents; the root is last).

    parent (n_nodes,) i64 (-1 for the root); level (n_nodes,) i64 (height: leaves 0); own_ptr / own
    (CSR): the DOFs each node eliminates, in elimination order; bnd_ptr / bnd: the node's boundary DOFs,
    sorted by elimination position; perm (n_free,): DOFs in elimination order; pos (n_dof,): position
    of each DOF in perm (-1 for eliminated PEC DOFs)."""
    parent: np.ndarray
    level: np.ndarray
    own_ptr: np.ndarray
    own: np.ndarray
    bnd_ptr: np.ndarray
    bnd: np.ndarray
    perm: np.ndarray
    pos: np.ndarray

    @property
    def n_nodes(self) -> int:
        return len(self.parent)

    def own_size(self) -> np.ndarray:
        return np.diff(self.own_ptr)

    def bnd_size(self) -> np.ndarray:
        return np.diff(self.bnd_ptr)

    def flops(self, complex_: bool = True) -> float:
        """Real floating-point operations of the partial LU of every front (complex: 4 per complex
        multiply-add pair, counted as 8 flops per complex FMA)."""
        e = self.own_size().astype(np.float64)
        b = self.bnd_size().astype(np.float64)
        # LU of the e x e block, the two triangular solves for the e x b panels, the b x b Schur update
        fma = e ** 3 / 3 + e ** 2 * b + e * b * b
        return float(fma.sum() * (8 if complex_ else 2))

    def factor_entries(self) -> int:
        """Entries of L and U kept for the solves: e^2 + 2 e b per front."""
        e = self.own_size().astype(np.int64)
        b = self.bnd_size().astype(np.int64)
        return int((e * e + 2 * e * b).sum())


def _split(cen: np.ndarray, tets: np.ndarray):
    """Bisect the tet list along the longest centroid axis at the widest gap near the median."""
    c = cen[:, tets]
    ext = c.max(axis=1) - c.min(axis=1)
    ax = int(np.argmax(ext))
    order = np.argsort(c[ax], kind="stable")
    v = c[ax, order]
    n = len(order)
    lo, hi = max(1, int(0.35 * n)), min(n - 1, int(0.65 * n))
    if hi <= lo:
        k = n // 2
    else:
        gaps = v[lo:hi + 1] - v[lo - 1:hi]
        # prefer the widest gap; among near-equal gaps the one closest to the median
        dist = np.abs(np.arange(lo, hi + 1) - n / 2) / n
        k = lo + int(np.argmax(gaps - 1e-9 * gaps.max() * dist))
    return tets[order[:k]], tets[order[k:]]


def nested_dissection(ent: np.ndarray, n_entity: int, cen: np.ndarray, free: np.ndarray, half: int,
                      leaf_tets: int = 64) -> EliminationTree:
    """Elimination tree of the Nedelec-2 system.

    ent (10, N_t) i64: each tet's entity ids (the first-kind DOFs, ``tet_to_field[:10]``); n_entity =
    H = N_e + N_f; cen (3, N_t): tet centroids; free (2 H,) bool: DOFs not eliminated by PEC; half = H
    (entity X owns DOFs X and X + H)."""
    nt = ent.shape[1]
    owner = np.full(n_entity, -1, dtype=np.int64)       # tree node that eliminates each entity
    stamp = np.full(n_entity, -1, dtype=np.int64)       # last node whose left half touched each entity
    nodes_tets: list[np.ndarray] = []
    nodes_own: list[np.ndarray] = []
    nodes_children: list[list[int]] = []
    # iterative preorder construction: (tets, parent id, which child)
    stack = [(np.arange(nt, dtype=np.int64), -1)]
    parent_pre: list[int] = []
    while stack:
        tets, par = stack.pop()
        nid = len(nodes_tets)
        nodes_tets.append(tets)
        parent_pre.append(par)
        nodes_children.append([])
        if par >= 0:
            nodes_children[par].append(nid)
        e = ent[:, tets]
        if len(tets) <= leaf_tets:
            u = np.unique(e)
            u = u[owner[u] < 0]
            owner[u] = nid
            nodes_own.append(u)
            continue
        left, right = _split(cen, tets)
        # separator: entities touched by both halves (stamped by the left half, met again on the right)
        stamp[ent[:, left]] = nid
        er_ = ent[:, right].ravel()
        sep = np.unique(er_[stamp[er_] == nid])
        sep = sep[owner[sep] < 0]
        owner[sep] = nid
        nodes_own.append(sep)
        stack.append((right, nid))
        stack.append((left, nid))
    n = len(nodes_tets)
    # postorder: children before parents
    post: list[int] = []
    visit = [(0, False)]
    while visit:
        v, done = visit.pop()
        if done:
            post.append(v)
            continue
        visit.append((v, True))
        for c in reversed(nodes_children[v]):
            visit.append((c, False))
    new_of_old = np.empty(n, dtype=np.int64)
    new_of_old[np.array(post)] = np.arange(n)
    # DOFs in elimination order: per node (postorder), each own entity's first then second-kind DOF
    own_dofs = []
    for old in post:
        u = nodes_own[old]
        d = np.stack([u, u + half], axis=1).reshape(-1)
        own_dofs.append(d[free[d]])
    own_ptr = np.zeros(n + 1, dtype=np.int64)
    own_ptr[1:] = np.cumsum([len(d) for d in own_dofs])
    perm = np.concatenate(own_dofs) if own_dofs else np.zeros(0, dtype=np.int64)
    pos = np.full(2 * half, -1, dtype=np.int64)
    pos[perm] = np.arange(len(perm))
    # boundary sets bottom-up: entities of the subtree's tets that hold an own entity, minus the
    # entities eliminated inside the subtree
    owner_new = np.where(owner >= 0, new_of_old[np.maximum(owner, 0)], -1)
    bnd_ent: list[np.ndarray] = [None] * n           # type: ignore[list-item]
    mark = np.zeros(n_entity, dtype=bool)            # reused: set for a node's own entities, then cleared
    parent = np.full(n, -1, dtype=np.int64)
    level = np.zeros(n, dtype=np.int64)
    for old in post:
        v = new_of_old[old]
        kids = [new_of_old[c] for c in nodes_children[old]]
        for c in kids:
            parent[c] = v
        tets = nodes_tets[old]
        own_u = nodes_own[old]
        if len(own_u):
            mark[own_u] = True
            touch = mark[ent[:, tets]].any(axis=0)
            mark[own_u] = False
            adj = np.unique(ent[:, tets[touch]])
        else:
            adj = np.zeros(0, dtype=np.int64)
        parts = [adj] + [bnd_ent[c] for c in kids]
        cand = np.unique(np.concatenate(parts))
        # keep ancestors only: entities eliminated after this node
        cand = cand[owner_new[cand] > v]
        bnd_ent[v] = cand
        level[v] = 1 + max((level[c] for c in kids), default=-1)
    bnd = []
    for v in range(n):
        u = bnd_ent[v]
        d = np.stack([u, u + half], axis=1).reshape(-1)
        d = d[free[d]]
        bnd.append(d[np.argsort(pos[d], kind="stable")])
    bnd_ptr = np.zeros(n + 1, dtype=np.int64)
    bnd_ptr[1:] = np.cumsum([len(d) for d in bnd])
    return EliminationTree(parent, level, own_ptr, perm, bnd_ptr,
                           np.concatenate(bnd) if bnd else np.zeros(0, dtype=np.int64), perm, pos)


@dataclass
class FrontStructure:
    """Flat arrays of the multifrontal factorization for a CSR pattern (what ``emfem_mf_create`` takes).

    Per front v (postorder): e[v] eliminated and b[v] boundary DOFs (front size n = e + b), parent[v]
    (-1 for the root) and level[v]; fdof[fdof_ptr[v]:fdof_ptr[v+1]]: the front's DOFs (own, then
    boundary); ea[ea_ptr[v]:ea_ptr[v] + b[v]]: the position of each boundary DOF in the parent's front;
    asm_slot / asm_off (sorted by front, asm_ptr): every CSR entry (i, j) of the free rows and columns
    goes to the front that eliminates the earlier of i and j, at local offset row + col * n."""
    n: int
    e: np.ndarray
    b: np.ndarray
    parent: np.ndarray
    level: np.ndarray
    fdof_ptr: np.ndarray
    fdof: np.ndarray
    ea_ptr: np.ndarray
    ea: np.ndarray
    asm_ptr: np.ndarray | None
    asm_slot: np.ndarray | None
    asm_off: np.ndarray | None
    tree: EliminationTree


def front_structure(tree: EliminationTree, indptr: np.ndarray | None, indices: np.ndarray | None,
                    with_lists: bool = True) -> FrontStructure:
    """The front lists, extend-add maps and assembly lists of ``tree`` for the CSR pattern
    (indptr, indices) of the full system (PEC rows and columns are skipped).  Without ``with_lists`` the
    assembly lists are left empty (``asm_ptr`` None) for the device to build (``emfem_mf_build_lists``)."""
    T = tree
    nf = T.n_nodes
    e = T.own_size().astype(np.int64)
    b = T.bnd_size().astype(np.int64)
    n_front = e + b
    N = len(T.pos)
    own_start = T.own_ptr[:-1]
    node_of_pos = np.repeat(np.arange(nf), e)             # front that eliminates each position
    # the front's DOF lists: own then boundary
    fdof_ptr = np.zeros(nf + 1, dtype=np.int64)
    fdof_ptr[1:] = np.cumsum(n_front)
    fdof = np.empty(fdof_ptr[-1], dtype=np.int64)
    for v in range(nf):
        o0 = fdof_ptr[v]
        fdof[o0:o0 + e[v]] = T.own[T.own_ptr[v]:T.own_ptr[v + 1]]
        fdof[o0 + e[v]:fdof_ptr[v + 1]] = T.bnd[T.bnd_ptr[v]:T.bnd_ptr[v + 1]]
    # boundary positions as sorted keys front * (N + 1) + pos: local index of a boundary DOF of front v
    bpos = T.pos[T.bnd]
    bfront = np.repeat(np.arange(nf), b)
    bkeys = bfront * (N + 1) + bpos

    def local_index(front: np.ndarray, dof: np.ndarray) -> np.ndarray:
        p = T.pos[dof]
        own = node_of_pos[p] == front
        out = np.empty(len(dof), dtype=np.int64)
        out[own] = p[own] - own_start[front[own]]
        nb = ~own
        if nb.any():
            k = np.searchsorted(bkeys, front[nb] * (N + 1) + p[nb])
            if (k >= len(bkeys)).any() or (bkeys[np.minimum(k, len(bkeys) - 1)] != front[nb] * (N + 1) + p[nb]).any():
                raise RuntimeError("front_structure: a DOF is in neither the own nor the boundary set of its front")
            out[nb] = e[front[nb]] + (k - T.bnd_ptr[front[nb]])
        return out

    # extend-add maps: each front's boundary DOFs in its parent's front
    ea_ptr = np.zeros(nf + 1, dtype=np.int64)
    ea_ptr[1:] = np.cumsum(b)
    has_par = T.parent[bfront] >= 0
    ea = np.full(len(T.bnd), -1, dtype=np.int64)
    ea[has_par] = local_index(T.parent[bfront[has_par]], T.bnd[has_par])
    if not with_lists:
        return FrontStructure(N, e.astype(np.int32), b.astype(np.int32), T.parent.astype(np.int32),
                              T.level.astype(np.int32), fdof_ptr, fdof.astype(np.int32), ea_ptr, ea.astype(np.int32),
                              None, None, None, T)
    # assembly lists from the CSR pattern (free rows and columns only)
    rows = np.repeat(np.arange(N, dtype=np.int64), np.diff(indptr))
    cols = indices.astype(np.int64)
    slot = np.arange(len(cols), dtype=np.int64)
    keep = (T.pos[rows] >= 0) & (T.pos[cols] >= 0)
    rows, cols, slot = rows[keep], cols[keep], slot[keep]
    pmin = np.minimum(T.pos[rows], T.pos[cols])
    front = node_of_pos[pmin]
    lr = local_index(front, rows)
    lc = local_index(front, cols)
    off = lr + lc * n_front[front]
    order = np.argsort(front, kind="stable")
    asm_ptr = np.zeros(nf + 1, dtype=np.int64)
    asm_ptr[1:] = np.cumsum(np.bincount(front, minlength=nf))
    return FrontStructure(N, e.astype(np.int32), b.astype(np.int32), T.parent.astype(np.int32),
                          T.level.astype(np.int32), fdof_ptr, fdof.astype(np.int32), ea_ptr, ea.astype(np.int32),
                          asm_ptr, slot[order].astype(np.int32), off[order].astype(np.int32), T)


class DeviceLU:
    """The device multifrontal LU of a :class:`~emerge_b200.sweep.FrequencySweep`'s system.

    The structure (ordering, fronts, assembly lists) is built once per mesh and PEC set; ``factor(f)``
    forms K_f = E − k0²B + Σ_p γ_p(k0) R_p on the device (``emfem_sweep_combine``; the Robin/port entries
    summed per CSR slot) and factors its equilibrated form.  ``precision`` is the arithmetic of the
    factorization: "c64" (complex64 fronts) or "c128" (complex128 fronts and update store, twice their
    memory, about half the speed); the factors the solves read are complex64 either way.  ``solve``
    applies (LU)⁻¹; the sweep uses it as the preconditioner of FP64 BiCGStab
    (:meth:`FrequencySweep.solve_lu`), also at neighbouring frequencies."""

    def __init__(self, sweep, leaf_tets: int = 64, precision: str = "c64"):
        import ctypes
        import time
        import torch
        from ._lib import Handle, check, lib, ptr
        from .sweep import _seg_from_keys
        t0 = time.perf_counter()
        P = sweep.problem
        mesh, fld = P.mesh, P.field
        self.sweep = sweep
        self.device = sweep.device
        H = mesh.n_edges + mesh.n_tris
        free = sweep.mask.cpu().numpy().astype(bool)
        cen = mesh.nodes[:, mesh.tets].mean(axis=1)
        self.tree = nested_dissection(fld.tet_to_field[:10], H, cen, free, H, leaf_tets=leaf_tets)
        S = front_structure(self.tree, None, None, with_lists=False)     # assembly lists: built on the device
        self.structure = S
        self.n_fronts = len(S.e)
        self.seconds_symbolic = time.perf_counter() - t0
        h = Handle.get(self.device)
        c = np.ascontiguousarray
        arrs = [c(S.e, np.int32), c(S.b, np.int32), c(S.parent, np.int32), c(S.level, np.int32),
                c(S.fdof_ptr, np.int64), c(S.fdof, np.int32), c(S.ea, np.int32)]
        p = ctypes.c_void_p()
        check(lib().emfem_mf_create(h.h, sweep.n, self.n_fronts, *[a.ctypes.data_as(ctypes.c_void_p) for a in arrs],
                                    None, None, None, ctypes.byref(p)), "emfem_mf_create")
        self._p = p
        check(lib().emfem_mf_build_lists(p, sweep.plan.nnz, ptr(sweep.plan.indptr), ptr(sweep.plan.indices)),
              "emfem_mf_build_lists")
        nb, fl, nl = ctypes.c_size_t(), ctypes.c_double(), ctypes.c_int()
        check(lib().emfem_mf_info(p, ctypes.byref(nb), ctypes.byref(fl), ctypes.byref(nl)), "emfem_mf_info")
        self.device_bytes, self.flops, self.n_levels = nb.value, fl.value, nl.value
        # Robin / port entries: CSR slot of every (row, port, col) patch entry, grouped by slot
        self._patch = None
        if sweep.n_ports:
            rp = sweep.patch_rowptr.cpu().numpy()
            rows = np.repeat(sweep.patch_rows.cpu().numpy().astype(np.int64), np.diff(rp))
            cols = sweep.patch_cols.cpu().numpy().astype(np.int64)
            slots = sweep.plan.find_slots(torch.from_numpy(rows), torch.from_numpy(cols)).cpu().numpy()
            if (slots < 0).any():
                raise RuntimeError("DeviceLU: a Robin entry lies outside the tet pattern")
            us, seg, idx = _seg_from_keys(slots)
            self._patch = (torch.from_numpy(us.astype(np.int32)).to(self.device),
                           torch.from_numpy(seg).to(self.device), torch.from_numpy(idx).to(self.device))
        self.frequency = None
        self.n_perturbed = 0
        self.precision = "c64"
        self.set_precision(precision)
        self.seconds_create = time.perf_counter() - t0
        self._reserved = 0

    def set_precision(self, precision: str) -> "DeviceLU":
        """Switch the factorization arithmetic ("c64" or "c128"); reallocates the workspace and drops the
        current factorization.  If the complex128 workspace does not fit, the LU stays complex64 and
        this raises."""
        from ._lib import check, lib
        if precision not in ("c64", "c128"):
            raise ValueError(f"DeviceLU: precision must be 'c64' or 'c128', not {precision!r}")
        if precision != self.precision:
            self.frequency = None
            check(lib().emfem_mf_set_precision(self._p, 128 if precision == "c128" else 64), "emfem_mf_set_precision")
            self.precision = precision
            import ctypes
            nb, fl, nl = ctypes.c_size_t(), ctypes.c_double(), ctypes.c_int()
            check(lib().emfem_mf_info(self._p, ctypes.byref(nb), ctypes.byref(fl), ctypes.byref(nl)), "emfem_mf_info")
            self.device_bytes = nb.value
        return self

    def __del__(self):
        p = getattr(self, "_p", None)
        if p is not None and p.value:
            try:
                import torch
                from ._lib import lib
                torch.cuda.synchronize(self.device)
                lib().emfem_mf_destroy(p)
            except Exception:
                pass
            self._p = None

    def operator_values(self, freq: float):
        """K_f values (nnz c128, device) on the plan pattern."""
        import torch
        from ._lib import Handle, check, lib, ptr
        from .ports import k0_of
        from .sweep import gather_sum
        sw = self.sweep
        k0 = k0_of(freq)
        K = torch.empty(sw.plan.nnz, dtype=torch.complex128, device=self.device)
        np_ = 0
        us = uv = None
        if self._patch is not None:
            us, seg, idx = self._patch
            g = torch.from_numpy(np.ascontiguousarray(sw.gammas([freq])[0])).to(self.device)
            scaled = sw.patch_vals * g[sw.patch_port.long()]
            uv = gather_sum(seg, idx, scaled)
            np_ = us.numel()
        h = Handle.get(self.device)
        check(lib().emfem_sweep_combine(h.h, sw.plan.nnz, ptr(sw.E), ptr(sw.B), k0 * k0, np_, ptr(us) if np_ else None,
                                        ptr(uv) if np_ else None, 1.0, 0.0, ptr(K)), "emfem_sweep_combine")
        return K

    def factor(self, freq: float) -> "DeviceLU":
        import ctypes
        import time
        import torch
        from ._lib import check, lib, ptr
        K = self.operator_values(freq)
        npert = ctypes.c_int()
        t0 = time.perf_counter()
        check(lib().emfem_mf_factor(self._p, ptr(K), ctypes.byref(npert)), "emfem_mf_factor")
        self.seconds_factor = time.perf_counter() - t0
        self.n_perturbed = npert.value
        self.frequency = freq
        return self

    def reserve(self, nrhs: int) -> None:
        from ._lib import check, lib
        if nrhs > self._reserved:
            check(lib().emfem_mf_reserve(self._p, nrhs), "emfem_mf_reserve")
            self._reserved = nrhs

    def solve(self, b):
        """(LU)⁻¹ b for b (N,) or (N, nrhs) complex128 on the device."""
        import torch
        from ._lib import check, lib, ptr
        b2 = b.reshape(b.shape[0], -1).to(device=self.device, dtype=torch.complex128).contiguous()
        self.reserve(b2.shape[1])
        x = torch.empty_like(b2)
        check(lib().emfem_mf_solve(self._p, b2.shape[1], ptr(b2), ptr(x)), "emfem_mf_solve")
        return x.reshape(b.shape)


def _main(argv=None) -> None:
    """``python -m emerge_b200.direct --cavity N`` (or ``--substrate NX NY NZ``): build the N³
    dielectric-loaded cavity's (or the substrate box's) sweep, factor its system at one frequency in the
    given precision, apply the LU to that frequency's right-hand side once, optionally (``--refine``)
    solve that system to 1e-8 with the LU-preconditioned FP64 BiCGStab, and print the timings (one
    GPU)."""
    import argparse
    import json
    import time
    import torch
    from . import problems
    from .sweep import FrequencySweep
    ap = argparse.ArgumentParser()
    ap.add_argument("--cavity", type=int, default=16, help="hex grid size of the cavity (40: 384 000 tets)")
    ap.add_argument("--substrate", type=int, nargs=3, default=None, metavar=("NX", "NY", "NZ"),
                    help="the substrate box's hex grid instead of the cavity (40 30 26: 187 200 tets)")
    ap.add_argument("--freq-index", type=int, default=50, help="index into the problem's frequency list")
    ap.add_argument("--precision", default="c64", choices=["c64", "c128"], help="factorization arithmetic")
    ap.add_argument("--refine", action="store_true", help="also solve the system to 1e-8 (LU-preconditioned)")
    a = ap.parse_args(argv)
    P = problems.substrate_box(*a.substrate) if a.substrate else problems.cavity(n=a.cavity)
    sw = FrequencySweep(P)
    f = float(P.freqs[min(a.freq_index, len(P.freqs) - 1)])
    lu = DeviceLU(sw, precision=a.precision).factor(f)
    b = sw.rhs([(f, 0)])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lu.solve(b)
    torch.cuda.synchronize()
    t_solve = time.perf_counter() - t0
    out = {"tets": int(P.mesh.n_tets), "dof": int(sw.n), "freq": f, "precision": a.precision,
           "fronts": lu.n_fronts, "levels": lu.n_levels, "factor_seconds": lu.seconds_factor, "flops": lu.flops,
           "device_gb": lu.device_bytes / 1e9, "solve_seconds": t_solve, "perturbed_pivots": lu.n_perturbed}
    if a.refine:
        r = sw.solve_lu([(f, 0)], lu, tol=1e-8, maxit=200)
        out.update(refined_status=int(r.status[0]), refined_iters=int(r.iters[0]), refined_relres=float(r.relres[0]))
    print(json.dumps(out))


if __name__ == "__main__":
    _main()
