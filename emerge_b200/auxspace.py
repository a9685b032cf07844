"""Auxiliary nodal space and the learned auxiliary-space preconditioner (``emfem_aux_*``, ``emfem_mpnn_*``).

The reference factorises every frequency directly (``SolverSuperLU``,
``src/emerge/_emerge/solver.py:535-572``) and has no preconditioner.  The device Krylov sweep uses

    M r = BJ r + G N(D_a⁻¹ Gᵀ r)

with BJ the DOF-pair block Jacobi, G the exact discrete gradient from the second-order nodal space
(mesh vertices and edges) into the Nédélec-2 basis, D_a = diag(Gᵀ K G) per system, and N either the
identity (``precond="aux"``) or the message-passing network trained here (``precond="learned"``).

:class:`AuxSpace` owns the device objects; :class:`Network` holds the parameters and wraps the
hand-written forward/backward/Adam kernels; :func:`train` fits the network on residual/correction
pairs that the sweep's own solves produce.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from ._lib import Handle, check, lib, ptr

__all__ = ["AuxSpace", "Network", "TrainReport", "make_pairs", "train"]

CHANNELS, LAYERS = 32, 4
NPARAMS = 2 * CHANNELS + LAYERS * 4 * CHANNELS * CHANNELS + 2 * CHANNELS


def _dev_i64(a, dev):
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=torch.int64).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).to(dev)


def _dev_f64(a, dev):
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=torch.float64).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)


class AuxSpace:
    """Discrete gradient G, Gᵀ, the vertex-edge incidence graph and the aux operator diagonals."""

    def __init__(self, mesh, device=None):
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = dev
        self.n_nodes, self.n_edges, self.n_tris = mesh.nodes.shape[1], mesh.edges.shape[1], mesh.tris.shape[1]
        self.n_field = 2 * (self.n_edges + self.n_tris)
        self._keep = [_dev_i64(mesh.edges, dev), _dev_i64(mesh.tris, dev), _dev_i64(mesh.tri_to_edge, dev),
                      _dev_f64(mesh.edge_lengths, dev)]
        h = Handle.get(dev)
        a = ctypes.c_void_p()
        check(lib().emfem_aux_create(h.h, self.n_nodes, self.n_edges, self.n_tris, *[ptr(t) for t in self._keep],
                                     ctypes.byref(a)), "emfem_aux_create")
        self._a = a
        na, ngt, ngr = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().emfem_aux_info(a, ctypes.byref(na), ctypes.byref(ngt), ctypes.byref(ngr)), "emfem_aux_info")
        self.n_aux, self.nnz_gt, self.nnz_graph = na.value, ngt.value, ngr.value
        self.n_ports = 0
        self.mask = None
        self._params = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._a

    def __del__(self):
        a = getattr(self, "_a", None)
        if a is not None and a.value:
            try:
                torch.cuda.synchronize(self.device)
                lib().emfem_aux_destroy(a)
            except Exception:
                pass
            self._a = None

    def export(self) -> dict:
        """G (ELL), Gᵀ (CSR) and the incidence graph as device tensors."""
        d = self.device
        out = dict(gcol=torch.empty((self.n_field, 6), dtype=torch.int32, device=d),
                   gval=torch.empty((self.n_field, 6), dtype=torch.float64, device=d),
                   gt_ptr=torch.empty(self.n_aux + 1, dtype=torch.int32, device=d),
                   gt_row=torch.empty(self.nnz_gt, dtype=torch.int32, device=d),
                   gt_val=torch.empty(self.nnz_gt, dtype=torch.float64, device=d),
                   graph_ptr=torch.empty(self.n_aux + 1, dtype=torch.int32, device=d),
                   graph_nbr=torch.empty(self.nnz_graph, dtype=torch.int32, device=d))
        Handle.get(d)
        check(lib().emfem_aux_export(self._a, *[ptr(out[k]) for k in ("gcol", "gval", "gt_ptr", "gt_row", "gt_val",
                                                                       "graph_ptr", "graph_nbr")]), "emfem_aux_export")
        return out

    def set_rows(self, new_of_old: torch.Tensor, n_new: int, aux_group: torch.Tensor | None = None) -> None:
        """Move G onto the rows of a grouped multi-mesh system (``emfem_aux_set_rows``); the operator
        diagonals must be set again afterwards."""
        nd = new_of_old.to(self.device, torch.int64).contiguous()
        grp = None if aux_group is None else aux_group.to(self.device, torch.int32).contiguous()
        ng = 1 if grp is None else int(grp.max().item()) + 1
        Handle.get(self.device)
        check(lib().emfem_aux_set_rows(self._a, int(n_new), ptr(nd), ng, None if grp is None else ptr(grp)),
              "emfem_aux_set_rows")
        Handle.get(self.device).raise_on_device_status("emfem_aux_set_rows")
        self.n_field = int(n_new)
        self.mask = None

    def set_operator(self, sweep) -> torch.Tensor:
        """Aux diagonals of a FrequencySweep's operator; returns [dE | dB | dR_p ...] (complex)."""
        h = Handle.get(self.device)
        diag = torch.empty((2 + sweep.n_ports) * self.n_aux, dtype=torch.complex128, device=self.device)
        self.mask = torch.empty(self.n_aux, dtype=torch.uint8, device=self.device)
        check(lib().emfem_aux_set_operator(
            self._a, sweep.n, ptr(sweep.plan.indptr), ptr(sweep.plan.indices), ptr(sweep.E), ptr(sweep.B),
            sweep.patch_rows.numel(), ptr(sweep.patch_rows), ptr(sweep.patch_rowptr), ptr(sweep.patch_cols),
            ptr(sweep.patch_vals), ptr(sweep.patch_port), sweep.n_ports, ptr(sweep.mask), ptr(diag), ptr(self.mask)),
            "emfem_aux_set_operator")
        self.n_ports = sweep.n_ports
        return diag

    def reserve(self, nsys: int) -> None:
        Handle.get(self.device)
        check(lib().emfem_aux_reserve(self._a, int(nsys)), "emfem_aux_reserve")

    def set_network(self, params: torch.Tensor | None) -> None:
        self._params = params
        check(lib().emfem_aux_set_network(self._a, ptr(params) if params is not None else None),
              "emfem_aux_set_network")

    def dinv(self, k0sq: torch.Tensor, gamma: torch.Tensor) -> torch.Tensor:
        """(n_aux, nsys) 1/diag(Gᵀ K_s G) on usable aux nodes, 0 elsewhere."""
        nsys = k0sq.numel()
        out = torch.empty((self.n_aux, nsys), dtype=torch.complex128, device=self.device)
        Handle.get(self.device)
        check(lib().emfem_aux_dinv(self._a, nsys, ptr(k0sq), ptr(gamma) if gamma is not None else None, ptr(out)),
              "emfem_aux_dinv")
        return out

    def restrict(self, v: torch.Tensor, dinv: torch.Tensor | None = None) -> torch.Tensor:
        """dinv ⊙ Gᵀ v for v (n_field, nsys) complex128."""
        v = v.contiguous()
        nsys = v.shape[1]
        out = torch.empty((self.n_aux, nsys), dtype=torch.complex128, device=self.device)
        Handle.get(self.device)
        check(lib().emfem_aux_restrict(self._a, nsys, ptr(dinv) if dinv is not None else None, ptr(v), ptr(out)),
              "emfem_aux_restrict")
        return out

    def prolong(self, za: torch.Tensor, free_mask: torch.Tensor | None = None) -> torch.Tensor:
        """G za on free rows for za (n_aux, nsys) complex128."""
        za = za.contiguous()
        nsys = za.shape[1]
        out = torch.empty((self.n_field, nsys), dtype=torch.complex128, device=self.device)
        Handle.get(self.device)
        check(lib().emfem_aux_prolong(self._a, nsys, ptr(za), ptr(free_mask) if free_mask is not None else None,
                                      ptr(out), 0), "emfem_aux_prolong")
        return out


class Network:
    """Parameters (FP32, device) and the hand-written kernels of the aux-space message-passing
    network: 4 layers, 32 complex (64 real) channels, real weights, vertex/edge node types.

    ``init="jacobi"`` starts at w_out = 0, i.e. exactly the aux-space Jacobi correction."""

    def __init__(self, aux: AuxSpace, seed: int = 0, init: str = "jacobi", params: torch.Tensor | None = None):
        assert lib().emfem_mpnn_nparams() == NPARAMS
        self.aux = aux
        dev = aux.device
        if params is not None:
            self.params = params.to(device=dev, dtype=torch.float32).contiguous().clone()
        else:
            g = torch.Generator().manual_seed(seed)
            C = CHANNELS
            parts = [torch.randn(2 * C, generator=g) / C ** 0.5]
            for _ in range(LAYERS):
                parts.append(torch.eye(C).repeat(2, 1, 1).reshape(-1) * 0.5 + torch.randn(2 * C * C, generator=g) * 0.3 / C ** 0.5)
                parts.append(torch.eye(C).repeat(2, 1, 1).reshape(-1) * 0.5 + torch.randn(2 * C * C, generator=g) * 0.3 / C ** 0.5)
            w_out = torch.zeros(2 * C) if init == "jacobi" else torch.randn(2 * C, generator=g) / C
            parts.append(w_out)
            self.params = torch.cat(parts).to(dev, torch.float32).contiguous()
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self._ws = {}

    def _buffers(self, nsys: int):
        if nsys not in self._ws:
            a, s = ctypes.c_int64(), ctypes.c_int64()
            check(lib().emfem_mpnn_workspace_floats(self.aux.handle, nsys, ctypes.byref(a), ctypes.byref(s)),
                  "emfem_mpnn_workspace_floats")
            self._ws = {nsys: (torch.empty(a.value, dtype=torch.float32, device=self.aux.device),
                               torch.empty(s.value, dtype=torch.float32, device=self.aux.device))}
        return self._ws[nsys]

    def active(self) -> bool:
        """False when the output weights are all zero: the network is then exactly the skip term, i.e.
        the aux-space Jacobi, and the solvers apply that instead of running the layers."""
        return bool(self.params[-2 * CHANNELS:].abs().max().item() > 0)

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """za = N(x) for x (n_aux, nsys) complex64; keeps the activations for backward."""
        x = x.to(torch.complex64).contiguous()
        act, _ = self._buffers(x.shape[1])
        za = torch.empty_like(x)
        Handle.get(self.aux.device)
        check(lib().emfem_mpnn_forward(self.aux.handle, x.shape[1], ptr(self.params), ptr(x), ptr(act), ptr(za)),
              "emfem_mpnn_forward")
        self._x = x
        return za

    def infer(self, x: torch.Tensor) -> torch.Tensor:
        """za = N(x) through the tensor-core inference kernels the solver uses (TF32 inputs)."""
        x = x.to(torch.complex64).contiguous()
        work = torch.empty(2 * self.aux.n_aux * x.shape[1] * 2 * CHANNELS, dtype=torch.float32, device=x.device)
        za = torch.empty_like(x)
        Handle.get(self.aux.device)
        check(lib().emfem_mpnn_infer(self.aux.handle, x.shape[1], ptr(self.params), ptr(x), ptr(work), ptr(za)),
              "emfem_mpnn_infer")
        return za

    def backward(self, dza: torch.Tensor) -> torch.Tensor:
        """Parameter gradient for dza = dL/dRe(za) + i dL/dIm(za) of the last forward."""
        dza = dza.to(torch.complex64).contiguous()
        act, scratch = self._buffers(dza.shape[1])
        grad = torch.empty_like(self.params)
        Handle.get(self.aux.device)
        check(lib().emfem_mpnn_backward(self.aux.handle, dza.shape[1], ptr(self.params), ptr(self._x), ptr(act),
                                        ptr(dza), ptr(grad), ptr(scratch)), "emfem_mpnn_backward")
        return grad

    def adam(self, grad: torch.Tensor, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999,
             eps: float = 1e-8, weight_decay: float = 0.0) -> None:
        self.step += 1
        h = Handle.get(self.aux.device)
        check(lib().emfem_adam_step(h.h, self.params.numel(), ptr(self.params), ptr(grad), ptr(self.m), ptr(self.v),
                                    lr, beta1, beta2, eps, weight_decay, self.step), "emfem_adam_step")


@dataclass
class TrainReport:
    steps: int = 0
    pairs: int = 0
    seconds: float = 0.0
    loss_first: float = float("nan")
    loss_last: float = float("nan")
    loss_jacobi_heldout: float = float("nan")
    loss_learned_heldout: float = float("nan")
    history: list = field(default_factory=list)
    validation_iters_aux: int = -1        # total iterations on the validation systems, aux Jacobi
    validation_iters_learned: int = -1    # same with the kept network
    validation_by_scale: dict = field(default_factory=dict)   # output scale -> validation iterations
    output_scale: float = 1.0             # factor applied to w_out after validation
    accepted: bool = True                 # False: the network was reset to the aux Jacobi (w_out = 0)


def make_pairs(sweep, systems, snapshots=(8, 24, 64), tol: float = 1e-10, maxit: int = 20000):
    """Residual/correction pairs from the sweep's own solves: the plain block-Jacobi BiCGStab is
    stopped after k iterations (x_k), the same systems are solved to ``tol`` with the aux-space
    preconditioner (x*); each pair is (r_k = b - K x_k, e_k = x* - x_k) with its system.
    Returns a list of (system, r (n,), e (n,)) complex128 device tensors."""
    ref = sweep.solve(systems, tol=tol, maxit=maxit, precond="aux")
    b = sweep.rhs(systems)
    out = []
    for k in snapshots:
        res = sweep.solve(systems, tol=1e-30, maxit=k, precond="block_jacobi")
        r = b - sweep.apply(systems, res.x)
        r = r * sweep.mask[:, None]
        e = ref.x - res.x
        for j, sysj in enumerate(systems):
            if ref.status[j] == 0:
                out.append((sysj, r[:, j].clone(), e[:, j].clone()))
    return out


def _loss_and_grad(net: Network, aux: AuxSpace, sweep, batch, need_grad: bool = True):
    """L = mean_s ||G za_s - e_s||² / ||e_s||², za = N(D_a⁻¹ Gᵀ r_s): the aux correction should
    reproduce the gradient part of the true correction."""
    systems = [p[0] for p in batch]
    r = torch.stack([p[1] for p in batch], dim=1)
    e = torch.stack([p[2] for p in batch], dim=1)
    k0 = torch.from_numpy(sweep.k0sq([f for f, _ in systems])).to(aux.device)
    g = sweep.gammas([f for f, _ in systems])
    gam = torch.from_numpy(np.ascontiguousarray(np.stack([g.real, g.imag], -1).reshape(-1))).to(aux.device)
    dinv = aux.dinv(k0, gam)
    x = aux.restrict(r, dinv)
    za = net.forward(x.to(torch.complex64))
    diff = aux.prolong(za.to(torch.complex128), sweep.mask) - e
    en = (e.abs() ** 2).sum(dim=0)
    loss = float(((diff.abs() ** 2).sum(dim=0) / en).mean())
    if not need_grad:
        return loss, None
    dza = aux.restrict(diff * (2.0 / (en * len(batch)))[None, :])
    return loss, net.backward(dza)


def train(net: Network, sweep, pairs, heldout=None, steps: int = 200, batch: int = 8, lr: float = 1e-3,
          seed: int = 0, log_every: int = 20, validate=None, tol: float = 1e-8,
          scales=(1.0, 0.5, 0.25)) -> TrainReport:
    """Adam on the correction loss over random minibatches of pairs (all on the GPU).

    With ``validate`` (a list of held-out (frequency, port) systems), the learned term is scaled by
    each factor in ``scales`` (its output weights w_out times the factor) and by 0, which is
    exactly the aux-space Jacobi the network started from.  Each variant solves the validation systems,
    and the variant with the fewest iterations is kept.  ``accepted`` is False when that variant is 0.
    The correction loss does not always predict Krylov iterations on these indefinite systems, so
    this selection keeps a training run from ever slowing the solve down."""
    aux = net.aux
    rng = np.random.default_rng(seed)
    rep = TrainReport(pairs=len(pairs))
    t0 = time.perf_counter()
    for it in range(steps):
        idx = rng.choice(len(pairs), min(batch, len(pairs)), replace=False)
        loss, grad = _loss_and_grad(net, aux, sweep, [pairs[i] for i in idx])
        if it == 0:
            rep.loss_first = loss
        net.adam(grad, lr=lr)
        rep.loss_last = loss
        if it % log_every == 0:
            rep.history.append((it, loss))
    torch.cuda.synchronize(aux.device)
    rep.steps = steps
    rep.seconds = time.perf_counter() - t0
    if heldout:
        jac = Network(aux, init="jacobi")
        rep.loss_jacobi_heldout = float(np.mean([_loss_and_grad(jac, aux, sweep, [p], False)[0] for p in heldout]))
        rep.loss_learned_heldout = float(np.mean([_loss_and_grad(net, aux, sweep, [p], False)[0] for p in heldout]))
    if validate:
        prev = sweep.network
        rep.validation_iters_aux = int(sweep.solve(validate, tol=tol, maxit=40000, precond="aux").iters.sum())
        rep.validation_by_scale[0.0] = rep.validation_iters_aux
        w_out = net.params[-2 * CHANNELS:].clone()
        sweep.set_network(net)
        for a in scales:
            net.params[-2 * CHANNELS:] = w_out * a
            r = sweep.solve(validate, tol=tol, maxit=40000, precond="learned")
            rep.validation_by_scale[float(a)] = int(r.iters.sum()) if (r.status == 0).all() else 1 << 30
        sweep.set_network(prev)
        best = min(rep.validation_by_scale, key=lambda k: (rep.validation_by_scale[k], k))
        net.params[-2 * CHANNELS:] = w_out * best
        rep.output_scale = best
        rep.accepted = best > 0.0
        rep.validation_iters_learned = rep.validation_by_scale[best]
    return rep
