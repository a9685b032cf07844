"""Device-resident frequency sweep: assembly once, then batched Krylov solves of
K_f = E − k0_f²·B + Σ_p γ_p(k0_f)·R̂_p with port excitations b_{f,p} = s_p(k0_f)·b̂_p.

This is the GPU counterpart of ``Microwave3D.run_sweep`` → ``Assembler.assemble_freq_matrix`` →
``SimJob.iter_Ab`` → ``SolveRoutine.solve`` (``MW/microwave_3d.py:663-878``,
``ASM/assembler.py:189-429``, ``MW/simjob.py:82-107``, ``src/emerge/_emerge/solver.py:1241-1326``):

* E/B come from the fused plan assembly (``CsrPlan``) and are shared by every frequency;
* each port's Robin matrix is linear in γ (``ASM/robinbc.py:126-292``: Bmat·γ/(2A)²), so R̂_p is
  assembled once with γ = 1 and scaled per frequency inside the SpMV;
* the port force vector is linear in U_inc = s_p(k0)·shape (``MW/microwave_bc.py:864-883``), so b̂_p
  is assembled once from the unit mode shape;
* PEC DOFs (``ASM/assembler.py:274-307``) are a free-DOF mask, the exact equivalent of the
  reference's submatrix elimination.

``MW/`` = ``src/emerge/_emerge/physics/microwave/``; ``ASM/`` = ``MW/assembly/``.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import Handle, check, lib, ptr, ERR_NOT_CONVERGED
from .assembly import CsrPlan, DeviceMesh, dunavant4, tri_abc2_device, tri_robin_device
from .ports import k0_of

PRECOND = {"none": 0, "jacobi": 1, "block_jacobi": 2, "aux": 3, "learned": 4}
PRECISION = {"fp64": 0, "mixed": 1}
METHOD = {"cocg": 0, "bicgstab": 1}


def _seg_from_keys(keys: np.ndarray):
    """Stable grouping of equal keys: (unique_keys, seg (n_u+1), idx) with contributions in
    original order inside each group."""
    order = np.argsort(keys, kind="stable")
    ks = keys[order]
    first = np.ones(len(ks), dtype=bool)
    first[1:] = ks[1:] != ks[:-1]
    starts = np.flatnonzero(first)
    seg = np.append(starts, len(ks)).astype(np.int32)
    return ks[starts], seg, order.astype(np.int32)


def gather_sum(seg: torch.Tensor, idx: torch.Tensor, src: torch.Tensor) -> torch.Tensor:
    n_out = seg.numel() - 1
    out = torch.empty(n_out, dtype=torch.complex128, device=src.device)
    h = Handle.get(src.device)
    check(lib().emfem_segmented_gather_sum(h.h, n_out, ptr(seg), ptr(idx), ptr(src.contiguous()), ptr(out)),
          "emfem_segmented_gather_sum")
    return out


@dataclass
class SolveResult:
    x: torch.Tensor          # (N, nsys) complex128, device
    status: np.ndarray
    iters: np.ndarray
    relres: np.ndarray
    systems: list
    seconds: float
    fallbacks: int = 0       # systems re-solved by a fallback method


def sparam_corrections(S: np.ndarray, col: bool = True, single: bool = True, recip: bool = False) -> np.ndarray:
    """The reference's S-matrix post-corrections, defaults as in its settings
    (``MW/microwave_3d.py:1208-1225``, ``src/emerge/_emerge/settings.py:25-27``)."""
    S = np.array(S, dtype=np.complex128)
    N = S.shape[1]
    if recip:
        S = (S + S.T) / 2
    if col:
        for j in range(N):
            S[:, j] = S[:, j] / max(1.0, float(np.sum(np.abs(S[:, j]) ** 2)))
    if single:
        for i in range(N):
            for j in range(N):
                S[i, j] = S[i, j] / max(1.0, abs(S[i, j]))
    return S


class FrequencySweep:
    def __init__(self, problem, device=None, assemble: bool = True):
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = dev
        self.problem = problem
        fld, mesh = problem.field, problem.mesh
        self.dmesh = DeviceMesh(mesh, fld, dev)
        self.plan = CsrPlan(self.dmesh)
        self.n = self.plan.n_field
        self.er = torch.from_numpy(np.ascontiguousarray(problem.er)).to(dev)
        self.ur = torch.from_numpy(np.ascontiguousarray(problem.ur)).to(dev)
        self.E = self.B = None
        if assemble:
            self.assemble()
        self._build_ports()
        mask = np.ones(self.n, dtype=np.uint8)
        mask[problem.pec_ids] = 0
        self.mask = torch.from_numpy(mask).to(dev)
        self._ws = None
        self._aux = None
        self.network = None
        self._learned_active = False

    @classmethod
    def port_terms(cls, problem, device=None) -> "FrequencySweep":
        """A sweep object holding only the problem's port and Robin terms, port vectors and free-DOF
        mask, with no operator: what a batch of meshes whose operator is assembled elsewhere needs
        from each mesh (right-hand sides, Robin coefficients, S-parameters)."""
        fs = cls.__new__(cls)
        fs.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        fs.problem = problem
        fs.dmesh = DeviceMesh(problem.mesh, problem.field, fs.device)
        fs.n = problem.field.n_field
        fs.plan = None
        fs.E = fs.B = None
        fs._build_ports()
        mask = np.ones(fs.n, dtype=np.uint8)
        mask[problem.pec_ids] = 0
        fs.mask = torch.from_numpy(mask).to(fs.device)
        fs._ws = None
        fs._aux = None
        fs.network = None
        fs._learned_active = False
        return fs

    def aux_space(self):
        """The auxiliary nodal space of this mesh with this operator's diagonals (built once)."""
        if self._aux is None:
            from .auxspace import AuxSpace
            self._aux = AuxSpace(self.problem.mesh, self.device)
            self._aux.set_operator(self)
        return self._aux

    def set_network(self, net) -> None:
        """Use this trained :class:`auxspace.Network` for ``precond="learned"``.  A network whose output
        weights are zero (validation rejected the learned term) is the aux-space Jacobi exactly, and
        ``precond="learned"`` then runs that without the network's layers."""
        self.network = net
        self._learned_active = net is not None and net.active()
        self.aux_space().set_network(net.params if net is not None else None)

    def assemble(self):
        self.E, self.B = self.plan.assemble(self.er, self.ur, self.E, self.B)
        if getattr(self, "_aux", None) is not None:    # the aux diagonals follow the operator
            self._aux.set_operator(self)
        return self.E, self.B

    def _build_ports(self):
        P, fld, mesh, dev = self.problem, self.problem.field, self.problem.mesh, self.device
        dp = dunavant4()
        self.dpts = torch.from_numpy(dp).to(dev)
        N = self.n
        blocks_all, meta_rows, meta_cols, meta_port = [], [], [], []
        self.bhat = []
        robin = list(getattr(P, "robin", []) or [])
        off = 0
        for q, port in enumerate(P.ports):
            tid = np.asarray(port.tri_ids, dtype=np.int64)
            tn = mesh.tris[:, tid]
            v = mesh.nodes[:, tn]                                     # (3, 3, ns)
            pts = np.einsum("cvs,vp->cps", v, dp[1:4])                # (3, npts, ns)
            U = port.shape_global(pts[0], pts[1], pts[2]).astype(np.complex128)   # (3, npts, ns)
            blocks, bvec = tri_robin_device(self.dmesh, torch.from_numpy(np.ascontiguousarray(tn)).to(dev), 1.0,
                                            torch.from_numpy(np.ascontiguousarray(U)).to(dev), self.dpts)
            t2f = fld.tri_to_field[:, tid]                            # (8, ns)
            rows = np.repeat(t2f.T, 8, axis=1).ravel()                # entry 8a+b -> row t2f[a]
            cols = np.tile(t2f.T, (1, 8)).ravel()                     # col t2f[b]
            blocks_all.append(blocks.reshape(-1))
            meta_rows.append(rows); meta_cols.append(cols); meta_port.append(np.full(rows.shape, q))
            # port vector b̂_q: Bvec[tri_to_field[:, t]] += bvec[t] in triangle order
            dofs = t2f.T.ravel()
            ud, seg, idx = _seg_from_keys(dofs)
            vals = gather_sum(torch.from_numpy(seg).to(dev), torch.from_numpy(idx).to(dev), bvec.reshape(-1))
            bh = torch.zeros(N, dtype=torch.complex128, device=dev)
            bh[torch.from_numpy(ud).to(dev)] = vals
            self.bhat.append(bh)
            off += len(rows)
        # non-excited Robin boundaries: R̂ with γ = 1 (no excitation), as extra patch "ports"; a
        # second-order ABC adds its correction matrix (coefficient 1) as one more
        self._gamma_fns = [p.get_gamma for p in P.ports]
        for bc in robin:
            tid = np.asarray(bc.tri_ids, dtype=np.int64)
            tn = torch.from_numpy(np.ascontiguousarray(mesh.tris[:, tid])).to(dev)
            t2f = fld.tri_to_field[:, tid]
            parts = [(tri_robin_device(self.dmesh, tn, 1.0)[0], bc.get_gamma)]
            if getattr(bc, "order", 1) == 2:
                parts.append((tri_abc2_device(self.dmesh, tn, 1.0), bc.get_gamma2))
            for blocks, gfn in parts:
                q = len(self._gamma_fns)
                self._gamma_fns.append(gfn)
                blocks_all.append(blocks.reshape(-1))
                meta_rows.append(np.repeat(t2f.T, 8, axis=1).ravel())
                meta_cols.append(np.tile(t2f.T, (1, 8)).ravel())
                meta_port.append(np.full(8 * 8 * len(tid), q))
        nports = len(self._gamma_fns)
        if nports > 8:
            raise ValueError("at most 8 ports + Robin terms per sweep")
        if not meta_rows:                     # no ports and no Robin boundaries (a closed cavity)
            i32 = dict(dtype=torch.int32, device=dev)
            self.patch_vals = torch.zeros(0, dtype=torch.complex128, device=dev)
            self.patch_rows = torch.zeros(0, **i32)
            self.patch_rowptr = torch.zeros(1, **i32)
            self.patch_cols = torch.zeros(0, **i32)
            self.patch_port = torch.zeros(0, **i32)
            self.n_ports = 0
            return
        rows = np.concatenate(meta_rows); cols = np.concatenate(meta_cols); port = np.concatenate(meta_port)
        src = torch.cat(blocks_all)
        keys = (rows * nports + port) * N + cols
        uk, seg, idx = _seg_from_keys(keys)
        self.patch_vals = gather_sum(torch.from_numpy(seg).to(dev), torch.from_numpy(idx).to(dev), src)
        u_rows = uk // (nports * N)
        u_port = (uk // N) % nports
        u_cols = uk % N
        prow, pstart = np.unique(u_rows, return_index=True)
        self.patch_rows = torch.from_numpy(prow.astype(np.int32)).to(dev)
        self.patch_rowptr = torch.from_numpy(np.append(pstart, len(uk)).astype(np.int32)).to(dev)
        self.patch_cols = torch.from_numpy(u_cols.astype(np.int32)).to(dev)
        self.patch_port = torch.from_numpy(u_port.astype(np.int32)).to(dev)
        self.n_ports = nports

    # ---------------------------------------------------------------- S-parameters
    def _port_sp_data(self) -> list:
        """Per port: owning tets, node ids, unit mode shape at the quadrature points and the weight of the
        owning tet by mode type: 1/sqrt(mean diag ur / mean diag er) (TEM), 1/mean(diag ur) (TE),
        1/mean(diag er) (TM) (``_compute_s_data``, ``MW/microwave_3d.py:1295-1303``)."""
        if getattr(self, "_spdata", None) is not None:
            return self._spdata
        P, mesh, dev = self.problem, self.problem.mesh, self.device
        dp = dunavant4()
        out = []
        for port in P.ports:
            tid = np.asarray(port.tri_ids, dtype=np.int64)
            tn = mesh.tris[:, tid]
            owner = mesh.tri_to_tet[0, tid]
            pts = np.einsum("cvs,vp->cps", mesh.nodes[:, tn], dp[1:4])               # (3, npts, ntri)
            shape = port.shape_global(pts[0], pts[1], pts[2]).astype(np.complex128)
            ur, er = P.ur[:, :, owner], P.er[:, :, owner]
            mt = port.modetype(0.0) if hasattr(port, "modetype") else "TE"
            if mt == "TEM":
                const = 1.0 / np.sqrt((ur[0, 0] + ur[1, 1] + ur[2, 2]) / (er[0, 0] + er[1, 1] + er[2, 2]))
            elif mt == "TE":
                const = 1.0 / ((ur[0, 0] + ur[1, 1] + ur[2, 2]) / 3)
            else:
                const = 1.0 / ((er[0, 0] + er[1, 1] + er[2, 2]) / 3)
            const = np.asarray(const, dtype=np.complex128)
            out.append(dict(n=len(tid),
                            tri_tet=torch.from_numpy(np.ascontiguousarray(owner)).to(dev),
                            tri_nodes=torch.from_numpy(np.ascontiguousarray(tn)).to(dev),
                            shape=torch.from_numpy(np.ascontiguousarray(shape)).to(dev),
                            const=torch.from_numpy(np.ascontiguousarray(const)).to(dev)))
        self._spdata = out
        return out

    def port_overlaps(self, x: torch.Tensor) -> tuple[np.ndarray, np.ndarray]:
        """(overlap (n_ports, nsys), mode_norm (n_ports,)) of the solutions x (N, nsys) on every port face."""
        x = x.contiguous()
        nsys = x.shape[1]
        h = Handle.get(self.device)
        d_m = self.dmesh
        ov, nm = [], []
        for d in self._port_sp_data():
            work = torch.empty(d["n"] * (nsys + 1), dtype=torch.complex128, device=self.device)
            o = torch.empty(nsys, dtype=torch.complex128, device=self.device)
            m = torch.empty(1, dtype=torch.complex128, device=self.device)
            check(lib().emfem_port_overlap(h.h, d_m.n_nodes, ptr(d_m.nodes), d_m.n_tets, ptr(d_m.tets),
                                           ptr(d_m.tet_to_field), self.n, d["n"], ptr(d["tri_tet"]), ptr(d["tri_nodes"]),
                                           ptr(self.dpts), self.dpts.shape[1], ptr(d["shape"]), ptr(d["const"]), nsys,
                                           ptr(x), ptr(work), ptr(o), ptr(m)), "emfem_port_overlap")
            ov.append(o.cpu().numpy())
            nm.append(m.cpu().numpy()[0])
        h.raise_on_device_status("emfem_port_overlap")
        return np.array(ov), np.array(nm)

    def _lumped_lines(self, port) -> dict:
        """Voltage lines of a lumped port (``define_lumped_port_integration_points``,
        ``MW/microwave_3d.py:1432-1470``): from every port-face node of minimal projection on the
        port direction, 21 points over ``height`` along it; each point is assigned the last of the
        face tets (ascending, ``Mesh3D.get_face_tets``) that contains it, with the reference's
        inclusion test (``elements/ned2_interp.py:174-211``).  The composite 3-point Gauss rule of
        ``Line.line_integral`` (``coord.py:24-61, :149-153``) on equally spaced samples is Simpson's
        rule, so V = Σ_p w_p E(x_p)·dl with w = (1, 4, 2, ..., 4, 1)/3, averaged over the lines."""
        cache = getattr(self, "_lumped_cache", None)
        if cache is None:
            cache = self._lumped_cache = {}
        if id(port) in cache:
            return cache[id(port)]
        mesh, dev = self.problem.mesh, self.device
        tid = np.asarray(port.tri_ids, dtype=np.int64)
        nids = np.unique(mesh.tris[:, tid])
        dirv = np.asarray(port.direction, dtype=np.float64)
        xs, ys, zs = mesh.nodes[0, nids], mesh.nodes[1, nids], mesh.nodes[2, nids]
        dot = xs * dirv[0] + ys * dirv[1] + zs * dirv[2]
        start = np.flatnonzero(dot == np.min(dot))
        npl = 21
        lines_pts, lines_dl = [], []
        for k in start:
            p0 = np.array([xs[k], ys[k], zs[k]])
            p1 = p0 + dirv * port.height
            pts = np.stack([np.linspace(p0[i], p1[i], npl) for i in range(3)])
            lines_pts.append(pts)
            lines_dl.append(np.repeat((pts[:, 1] - pts[:, 0])[None, :], npl, axis=0))
        pts = np.concatenate(lines_pts, axis=1)
        dl = np.concatenate(lines_dl, axis=0)
        w1 = np.ones(npl)
        w1[1:-1:2] = 4.0
        w1[2:-1:2] = 2.0
        w = np.tile(w1 / 3.0, len(start)) / len(start)
        ftets = mesh.face_tets(tid)
        owner = np.full(pts.shape[1], -1, dtype=np.int64)
        for t in ftets:
            v = mesh.nodes[:, mesh.tets[:, t]]
            basis = np.linalg.inv(np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]], axis=1))
            loc = basis @ (pts - v[:, :1])
            inside = (loc.sum(axis=0) <= 1.00000001) & (loc >= -1e-6).all(axis=0)
            owner[inside] = t
        if (owner < 0).any():
            raise RuntimeError("lumped port: a voltage-line point lies in none of the port's face tets")
        d = dict(npts=pts.shape[1], w=w,
                 pts=torch.from_numpy(np.ascontiguousarray(pts)).to(dev),
                 dl=torch.from_numpy(np.ascontiguousarray(dl)).to(dev),
                 pt_tet=torch.from_numpy(owner).to(dev))
        cache[id(port)] = d
        return d

    def port_voltages(self, port, x: torch.Tensor) -> np.ndarray:
        """Lumped-port voltage V (nsys,) of the solutions x (N, nsys), E·dl on the device."""
        d = self._lumped_lines(port)
        x = x.contiguous()
        nsys = x.shape[1]
        out = torch.empty((d["npts"], nsys), dtype=torch.complex128, device=self.device)
        h = Handle.get(self.device)
        dm = self.dmesh
        check(lib().emfem_point_field_dot(h.h, dm.n_nodes, ptr(dm.nodes), dm.n_tets, ptr(dm.tets),
                                          ptr(dm.tet_to_field), self.n, d["npts"], ptr(d["pt_tet"]), ptr(d["pts"]),
                                          ptr(d["dl"]), nsys, ptr(x), ptr(out)), "emfem_point_field_dot")
        h.raise_on_device_status("emfem_point_field_dot")
        return d["w"] @ out.cpu().numpy()

    def sparams(self, res: SolveResult, corrections: bool = False) -> dict:
        """S-parameters of solved systems: {frequency: (n_ports, n_ports) complex S} with the columns of
        the excited ports filled (NaN elsewhere).  For a waveguide mode port S[q, p] is field_power /
        mode_power / sqrt(P_p) of the reference's ``_post_process`` (``MW/microwave_3d.py:1110-1247``);
        for a lumped port it is (b / a) / sqrt(P_p) with a = the port voltage √(2 P Z0) and b = V − a
        (excited) or V, V from the voltage lines (``:1271-1291``).  ``corrections`` applies the
        reference's default column-power and |S| <= 1 caps."""
        P = self.problem
        mode_ports = [q for q, port in enumerate(P.ports) if hasattr(port, "qmode")]
        ov = nm = None
        if mode_ports:
            ov, nm = self.port_overlaps(res.x)
        volts = {q: self.port_voltages(port, res.x) for q, port in enumerate(P.ports) if not hasattr(port, "qmode")}
        out: dict = {}
        for s, (f, p) in enumerate(res.systems):
            k0 = k0_of(f)
            S = out.setdefault(f, np.full((len(P.ports), len(P.ports)), np.nan + 0j))
            for q, port in enumerate(P.ports):
                if q in volts:
                    a = port.voltage
                    b = volts[q][s] - a if q == p else volts[q][s]
                    S[q, p] = (b / a) / np.sqrt(P.ports[p].power)
                    continue
                scale = port.qmode(k0) * port.polarization * port.amplitude()
                S[q, p] = (ov[q, s] / (scale * nm[q]) - (1.0 if q == p else 0.0)) / np.sqrt(P.ports[p].power)
        if corrections:
            out = {f: sparam_corrections(S) for f, S in out.items()}
        return out

    # ---------------------------------------------------------------- per-frequency data
    def k0sq(self, freqs) -> np.ndarray:
        return np.array([k0_of(f) ** 2 for f in freqs])

    def gammas(self, freqs) -> np.ndarray:
        """(nsys, n_ports) complex coefficients of every patch term (ports, then non-excited Robin
        boundaries and second-order ABC corrections) at every frequency."""
        return np.array([[complex(g(k0_of(f))) for g in self._gamma_fns] for f in freqs]).reshape(len(freqs), -1)

    def rhs(self, systems) -> torch.Tensor:
        """(N, nsys) right-hand sides b + port_vector[p] (``MW/simjob.py:88-92``, b = 0)."""
        cols = []
        for f, q in systems:
            s = self.problem.ports[q].uinc_scale(k0_of(f))
            cols.append(self.bhat[q] * s)
        return torch.stack(cols, dim=1).contiguous()

    def workspace(self, nsys: int, precision: int) -> torch.Tensor:
        sz = ctypes.c_size_t()
        check(lib().emfem_krylov_workspace_size(self.n, self.plan.nnz, nsys, precision, ctypes.byref(sz)),
              "emfem_krylov_workspace_size")
        if self._ws is None or self._ws.numel() < sz.value:
            self._ws = torch.empty(sz.value, dtype=torch.uint8, device=self.device)
        return self._ws

    FALLBACK = {("learned", "mixed"): [("learned", "fp64"), ("aux", "fp64"), ("block_jacobi", "fp64")],
                ("learned", "fp64"): [("aux", "fp64"), ("block_jacobi", "fp64")],
                ("aux", "mixed"): [("aux", "fp64"), ("block_jacobi", "fp64")],
                ("aux", "fp64"): [("block_jacobi", "fp64")],
                ("block_jacobi", "mixed"): [("block_jacobi", "fp64")]}

    def solve(self, systems, tol: float = 1e-8, maxit: int = 20000, precond: str = "block_jacobi",
              precision: str = "fp64", method: str = "bicgstab", x0: torch.Tensor | None = None,
              raise_on_fail: bool = False, fallback: bool = False) -> SolveResult:
        """Solve the listed (frequency, port index) systems in one batched Krylov call (<= 64).

        With ``fallback``, systems that miss the tolerance are solved again, warm-started from where
        they stopped, by the next entry of ``FALLBACK[(precond, precision)]`` (learned -> aux-space
        Jacobi -> plain block Jacobi, mixed -> FP64); the FP64 true residual decides.  ``iters`` and
        ``seconds`` then include every attempt, and ``fallbacks`` counts the systems re-solved."""
        res = self._solve(systems, tol, maxit, precond, precision, method, x0, raise_on_fail and not fallback)
        if not fallback:
            return res
        for pc, pr in self.FALLBACK.get((precond, precision), []):
            bad = np.flatnonzero(res.status != 0)
            if len(bad) == 0:
                break
            if pc == "learned" and self.network is None:
                continue
            sub = [systems[j] for j in bad]
            r2 = self._solve(sub, tol, maxit, pc, pr, method, res.x[:, bad].contiguous(), False)
            res.x[:, bad] = r2.x
            res.status[bad] = r2.status
            res.iters[bad] += r2.iters
            res.relres[bad] = r2.relres
            res.seconds += r2.seconds
            res.fallbacks += len(bad)
        if raise_on_fail and (res.status != 0).any():
            raise RuntimeError(f"not converged after fallbacks: status {res.status}")
        return res

    def _solve(self, systems, tol, maxit, precond, precision, method, x0, raise_on_fail) -> SolveResult:
        freqs = [f for f, _ in systems]
        return self.solve_rhs(self.k0sq(freqs), self.rhs(systems), self.gammas(freqs), tol=tol, maxit=maxit,
                              precond=precond, precision=precision, method=method, x0=x0,
                              raise_on_fail=raise_on_fail, systems=systems)

    def solve_partitioned(self, systems, solver: str = "krylov", window: int = 5, world_size: int | None = None,
                          rank: int | None = None, return_x: bool = False, **kw) -> list[dict]:
        """Solve ``systems`` split across the ranks of the process group (one GPU each), as the reference's
        frequency-parallel sweep does (``MW/microwave_3d.py:795-861``): ``solver="krylov"`` deals the
        systems round-robin and solves each rank's share in batches of 64 (``solve``, keyword arguments
        passed on); ``solver="direct"`` deals whole windows of ``window`` consecutive frequencies (one
        factorization each, ``solve_direct``), balanced by their system count.  Returns, on every rank and
        in the order of ``systems``, one dict per system: status, iterations, FP64 relative residual and,
        with ``return_x``, the solution as a host array."""
        from . import distributed
        ws, rk = distributed.world()
        ws = ws if world_size is None else world_size
        rk = rk if rank is None else rank
        systems = list(systems)

        def pack(res, j):
            d = {"status": int(res.status[j]), "iters": int(res.iters[j]), "relres": float(res.relres[j])}
            if return_x:
                d["x"] = res.x[:, j].cpu().numpy()
            return d

        if solver == "krylov":
            def run(batch):
                r = self.solve(batch, **kw)
                return [pack(r, j) for j in range(len(batch))]
            return distributed.run_partitioned(systems, run, ws, rk, batch=64)
        if solver != "direct":
            raise ValueError("solver must be 'krylov' or 'direct'")
        freqs = sorted({f for f, _ in systems})
        wins = [freqs[i:i + window] for i in range(0, len(freqs), window)]
        members = [[j for j, (f, _) in enumerate(systems) if f in set(w)] for w in wins]

        def run_windows(batch):
            out = []
            for idx in batch:
                r = self.solve_direct([systems[j] for j in idx], window=window, **kw)
                out.append([(j, pack(r, q)) for q, j in enumerate(idx)])
            return out
        per_win = distributed.run_partitioned(members, run_windows, ws, rk, batch=1,
                                              cost=[len(m) for m in members])
        result: list = [None] * len(systems)
        for lst in per_win:
            for j, d in lst:
                result[j] = d
        return result

    def direct_solver(self, leaf_tets: int = 64):
        """The device multifrontal LU of this sweep's mesh (built once, on first use)."""
        if getattr(self, "_lu", None) is None:
            from .direct import DeviceLU
            self._lu = DeviceLU(self, leaf_tets=leaf_tets)
        return self._lu

    def solve_direct(self, systems, window: int = 5, tol: float = 1e-8, maxit: int = 400, adaptive: bool = False,
                     iter_band: tuple = (20, 40), max_window: int = 15, precision: str = "c64",
                     probe_maxit: int = 60) -> SolveResult:
        """Every listed (frequency, port) system through the device LU, the GPU counterpart of the
        reference's direct solve per frequency (``SolverSuperLU``, LU reused across the ports of a
        frequency, ``MW/simjob.py:82-107``).  The distinct frequencies, ascending, are cut into windows of
        ``window`` consecutive ones; each window's middle frequency is factored and all systems of the
        window are solved together by FP64 BiCGStab preconditioned with that factorization (at the
        factored frequency a couple of refinement steps, at its neighbours a Krylov solve of the shifted
        operator).  With ``adaptive``, each window's width follows the previous one's largest iteration
        count: wider by 2 below ``iter_band[0]``, narrower by 2 above ``iter_band[1]`` (between 3 and
        ``max_window``), since the shifted systems at a window's edges need more iterations where the
        cavity's modes are denser.

        ``precision`` is the factorization's arithmetic: "c64", "c128", or "auto": each window is first
        tried with a complex64 factorization and at most ``probe_maxit`` iterations; the systems it leaves
        unconverged are solved again from a complex128 factorization at the same frequency (at low
        frequency the near-null gradient space makes K ill-conditioned enough that complex64 fronts give
        no usable preconditioner).  After a complex128 window that needed fewer than ``iter_band[0]``
        iterations, the next window tries complex64 again.  If the complex128 workspace does not fit on
        the device, the complex64 results stand (status shows what did not converge), the window log
        records the failed switch, and the rest of the sweep stays complex64.  Results come back in the order of
        ``systems``; ``windows`` on the result lists (factored frequency, precision, systems, factor
        seconds, solve seconds, iterations) per attempt."""
        if precision not in ("c64", "c128", "auto"):
            raise ValueError(f"solve_direct: precision must be 'c64', 'c128' or 'auto', not {precision!r}")
        lu = self.direct_solver()
        freqs = sorted({f for f, _ in systems})
        n = len(systems)
        x = torch.zeros((self.n, n), dtype=torch.complex128, device=self.device)
        status = np.zeros(n, dtype=np.int64)
        iters = np.zeros(n, dtype=np.int64)
        relres = np.zeros(n)
        t0 = time.perf_counter()
        log = []
        w0, W = 0, window
        first = "c128" if precision == "c128" else "c64"
        c128_fits = True
        while w0 < len(freqs):
            wf = freqs[w0:w0 + W]
            w0 += len(wf)
            fw = set(wf)
            todo = [j for j, (f, _) in enumerate(systems) if f in fw]
            fc = wf[len(wf) // 2]
            imax = 0
            if precision != "auto" or first == "c128":
                attempts = [first]
            else:
                attempts = ["c64", "c128"] if c128_fits else ["c64"]
            for prec in attempts:
                if not todo:
                    break
                last = prec == attempts[-1]
                imax = 0                          # the window width follows the attempt that finished it
                try:
                    lu.set_precision(prec)
                except RuntimeError as exc:
                    if precision != "auto":
                        raise
                    # the complex128 workspace does not fit: the complex64 results stand
                    c128_fits, first = False, "c64"
                    log.append(dict(factored=fc, precision=prec, systems=len(todo), error=str(exc)))
                    break
                tf = time.perf_counter()
                lu.factor(fc)
                tf = time.perf_counter() - tf
                it_cap = maxit if last else min(maxit, probe_maxit)
                left = []
                for c0 in range(0, len(todo), 64):
                    sub = todo[c0:c0 + 64]
                    r = self.solve_lu([systems[j] for j in sub], lu, tol=tol, maxit=it_cap)
                    ok = (r.status == 0) & (r.relres <= tol)
                    x[:, sub] = r.x
                    status[sub] = r.status
                    iters[sub] = r.iters
                    relres[sub] = r.relres
                    left += [sub[i] for i in range(len(sub)) if not ok[i]]
                    log.append(dict(factored=fc, precision=prec, systems=len(sub), factor_seconds=tf,
                                    solve_seconds=r.seconds, iters=r.iters.tolist(), perturbed=lu.n_perturbed))
                    tf = 0.0
                    conv = r.iters if last else r.iters[ok]
                    imax = max(imax, int(conv.max()) if conv.size else it_cap)
                todo = [] if last else left
                if precision == "auto":
                    if prec == "c128":
                        first = "c64" if imax < iter_band[0] else "c128"
                    elif left and c128_fits:
                        first = "c128"
            if adaptive:
                if imax > iter_band[1] and W > 3:
                    W = max(3, W - 2)
                elif imax < iter_band[0] and W < max_window:
                    W = min(max_window, W + 2)
        res = SolveResult(x, status, iters, relres, list(systems), time.perf_counter() - t0)
        res.windows = log
        return res

    def solve_lu(self, systems, lu, tol: float = 1e-8, maxit: int = 500, x0: torch.Tensor | None = None,
                 raise_on_fail: bool = False) -> SolveResult:
        """The listed (frequency, port) systems by FP64 BiCGStab right-preconditioned with the device LU
        ``lu`` (:class:`~emerge_b200.direct.DeviceLU`, factored at one frequency of this sweep: at that
        frequency a few iterations refine its complex64 solution to the FP64 tolerance, at neighbouring
        ones the LU is a preconditioner for the shifted operator)."""
        freqs = [f for f, _ in systems]
        return self.solve_rhs(self.k0sq(freqs), self.rhs(systems), self.gammas(freqs), tol=tol, maxit=maxit,
                              x0=x0, raise_on_fail=raise_on_fail, systems=systems, lu=lu)

    def solve_rhs(self, k0sq, b: torch.Tensor, gammas=None, tol: float = 1e-8, maxit: int = 20000,
                  precond: str = "block_jacobi", precision: str = "fp64", method: str = "bicgstab",
                  x0: torch.Tensor | None = None, raise_on_fail: bool = False, systems=None, lu=None) -> SolveResult:
        """(E - k0sq_s B + sum_p gammas[s, p] R_p) x_s = b_s for arbitrary right-hand sides b (N, nsys)
        on the free DOFs (gammas default 0: the Robin terms drop out).  With ``lu`` (a factored
        :class:`~emerge_b200.direct.DeviceLU`) the solve is FP64 BiCGStab preconditioned by it."""
        b = b.to(device=self.device, dtype=torch.complex128).contiguous()
        nsys = b.shape[1]
        assert 1 <= nsys <= 64
        k0 = np.asarray(k0sq, dtype=np.float64).reshape(-1)
        g = np.zeros((nsys, self.n_ports), dtype=np.complex128) if gammas is None else np.asarray(gammas)
        gam = np.ascontiguousarray(np.stack([g.real, g.imag], axis=-1).reshape(-1))
        if gam.size == 0:
            gam = np.zeros(2)
        x = torch.zeros_like(b) if x0 is None else x0.clone().contiguous()
        prec = PRECISION[precision]
        ws = self.workspace(nsys, prec)
        status = (ctypes.c_int * nsys)()
        iters = (ctypes.c_int * nsys)()
        relres = (ctypes.c_double * nsys)()
        k0a = (ctypes.c_double * nsys)(*k0)
        ga = (ctypes.c_double * len(gam))(*gam)
        aux = None
        pc = PRECOND[precond]
        if pc >= 3 and lu is None:
            if precond == "learned" and self.network is None:
                raise ValueError("precond='learned' needs a trained network (FrequencySweep.set_network)")
            if pc == 4 and not self._learned_active:
                pc = PRECOND["aux"]            # zero output weights: the same operator, no layers to run
            a = self.aux_space()
            a.reserve(nsys)
            aux = a.handle
        h = Handle.get(self.device)
        if lu is not None:
            if lu.frequency is None:
                raise ValueError("solve_rhs: the LU has not been factored")
            lu.reserve(1 << (nsys - 1).bit_length())
            ws = self.workspace(nsys, 0)
            t0 = time.perf_counter()
            st = lib().emfem_krylov_solve_lu(h.h, self.n, self.plan.nnz, ptr(self.plan.indptr), ptr(self.plan.indices),
                                             ptr(self.E), ptr(self.B), nsys, k0a, self.patch_rows.numel(),
                                             ptr(self.patch_rows), ptr(self.patch_rowptr), ptr(self.patch_cols),
                                             ptr(self.patch_vals), ptr(self.patch_port), self.n_ports, ga, ptr(self.mask),
                                             ptr(b), ptr(x), tol, maxit, lu._p, ptr(ws), ws.numel(), status, iters, relres)
            dt = time.perf_counter() - t0
            if st not in (0, ERR_NOT_CONVERGED) or (raise_on_fail and st != 0):
                check(st, "emfem_krylov_solve_lu")
            return SolveResult(x, np.array(status[:]), np.array(iters[:]), np.array(relres[:]),
                               list(systems) if systems is not None else [], dt)
        t0 = time.perf_counter()
        st = lib().emfem_krylov_solve(h.h, METHOD[method], self.n, self.plan.nnz, ptr(self.plan.indptr), ptr(self.plan.indices),
                                    ptr(self.E), ptr(self.B), nsys, k0a,
                                    self.patch_rows.numel(), ptr(self.patch_rows), ptr(self.patch_rowptr),
                                    ptr(self.patch_cols), ptr(self.patch_vals), ptr(self.patch_port), self.n_ports, ga,
                                    ptr(self.mask), ptr(b), ptr(x), tol, maxit, pc, prec,
                                    ptr(ws), ws.numel(), status, iters, relres, aux)
        dt = time.perf_counter() - t0
        if st not in (0, ERR_NOT_CONVERGED) or (raise_on_fail and st != 0):
            check(st, "emfem_krylov_solve")
        return SolveResult(x, np.array(status[:]), np.array(iters[:]), np.array(relres[:]),
                           list(systems) if systems is not None else [], dt)

    def apply(self, systems, x: torch.Tensor) -> torch.Tensor:
        """y = K_f x for each system (FP64; PEC rows/cols eliminated)."""
        nsys = len(systems)
        freqs = [f for f, _ in systems]
        k0 = torch.from_numpy(self.k0sq(freqs)).to(self.device)
        g = self.gammas(freqs)
        gam = torch.from_numpy(np.ascontiguousarray(np.stack([g.real, g.imag], axis=-1).reshape(-1))).to(self.device)
        S = 1 << (nsys - 1).bit_length()          # the kernel takes a power-of-two batch
        if S != nsys:
            pad = S - nsys
            x = torch.cat([x, torch.zeros((x.shape[0], pad), dtype=x.dtype, device=x.device)], dim=1)
            k0 = torch.cat([k0, k0[-1:].repeat(pad)])
            gam = torch.cat([gam, gam[-2 * self.n_ports:].repeat(pad)]) if self.n_ports else gam
        y = torch.empty_like(x)
        h = Handle.get(self.device)
        check(lib().emfem_sweep_spmv(h.h, self.n, ptr(self.plan.indptr), ptr(self.plan.indices), ptr(self.E),
                                     ptr(self.B), S, ptr(k0), self.patch_rows.numel(), ptr(self.patch_rows),
                                     ptr(self.patch_rowptr), ptr(self.patch_cols), ptr(self.patch_vals),
                                     ptr(self.patch_port), self.n_ports, ptr(gam), ptr(self.mask), ptr(x.contiguous()),
                                     ptr(y)), "emfem_sweep_spmv")
        return y[:, :nsys] if S != nsys else y
