"""Benchmark: Nédélec-2 tets assembled/s (fused integrator + deterministic CSR scatter of E and B)
on the dielectric-loaded cavity (40³ hex grid × 6 = 384 000 tets, 2 480 240 DOF), plus the
frequency-sweep solves/s of the learned auxiliary-space preconditioner against plain block Jacobi
(BiCGStab to FP64 relative residual 1e-8) on the port-loaded waveguide sweep, and bounded-iteration
runs on the cavity.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--no-sweep]

One JSON line on rank 0.  Under torchrun every rank assembles its own copy of the mesh
(replicas: the path has no exchange step), timed on the device; the step time is the max over
ranks and ``value`` counts the tets of all ranks.  ``--impl reference`` times the CPU oracle (a
restatement of the reference's numba integrator plus SciPy's COO→CSR) on the host's cores.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Nedelec-2 tets assembled/s"
UNIT = "tets/s"
L2_BYTES = 126 * 2 ** 20
# assemble_chunk_kernel DRAM traffic per tet, ncu capture at 82 944 tets: (686 + 178) MB / 82 944
ASM_TRAFFIC_PER_TET = (686e6 + 178e6) / 82944


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the timed region."""
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"
    PERIOD_MS = 100

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.n0 = 0
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        # the timed region starts only once the sampler is producing rows
        t0 = time.perf_counter()
        while self.proc is not None and time.perf_counter() - t0 < 10.0 and self.proc.poll() is None:
            self.n0 = len(self._rows())
            if self.n0 > 0:
                break
            time.sleep(0.02)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(1.5 * self.PERIOD_MS / 1e3)      # one more sample as the region ends
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def _rows(self) -> list:
        rows = []
        if self.path and os.path.exists(self.path):
            with open(self.path) as fh:
                for line in fh:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        return rows

    def summary(self) -> dict:
        rows = self._rows()
        if self.path and os.path.exists(self.path):
            os.unlink(self.path)
        # rows written after the region started (the row the start waited for is before it)
        rows = rows[self.n0:] or rows[-1:]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows), "period_ms": self.PERIOD_MS}


def dist_init(gpus: int):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v: float) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(problem, seconds_target: float = 15.0) -> dict:
    """The CPU oracle (restated reference integrator + SciPy COO->CSR) on a prefix sample of tets."""
    import oracle
    from scipy.sparse import coo_matrix
    cores = len(os.sched_getaffinity(0))
    oracle.set_threads(cores)
    m, f = problem.mesh, problem.field
    nt = m.n_tets
    n = f.n_field

    def run(k):
        t0 = time.perf_counter()
        dE, dB, r, c = oracle.matrix_builder(m.nodes, m.tets[:, :k], m.tris, m.edges, m.edge_lengths,
                                             f.tet_to_field[:, :k], m.tet_to_edge[:, :k], problem.ur[:, :, :k],
                                             problem.er[:, :, :k])
        coo_matrix((dE, (r, c)), shape=(n, n)).tocsr()
        coo_matrix((dB, (r, c)), shape=(n, n)).tocsr()
        return time.perf_counter() - t0

    k = min(nt, 20000)
    dt = run(k)
    # grow the sample to ~seconds_target of work (bounded by the full mesh)
    k2 = int(min(nt, max(k, k * seconds_target / max(dt, 1e-3))))
    if k2 > k:
        k, dt = k2, run(k2)
    return {"value": k / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first {k} of {nt} tets: oracle _matrix_builder restatement (OpenMP) + SciPy coo->csr of E and B"}


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from emerge_b200 import problems
    P = problems.cavity()
    t_all = []
    cb = None
    # each step a bounded sample, sized so the whole run stays near two and a half minutes
    per_step = max(1.0, min(8.0, 150.0 / (args.warmup + args.steps)))
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(P, seconds_target=per_step)
        if i >= args.warmup:
            t_all.append(cb["value"])
    v = float(np.mean(t_all))
    cb["value"] = v
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "c128",
           "data": "synthetic", "config": workload_config(P), "cpu_baseline": cb,
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def workload_config(P) -> dict:
    g = round((P.mesh.n_tets / 6) ** (1 / 3))
    return {"workload": f"dielectric-loaded cavity, {g}x{g}x{g} hex grid x6 tets, 8 seeded eps blocks, Nedelec-2 c128",
            "n_tets": int(P.mesh.n_tets), "n_dof": int(P.field.n_field), "frequencies": int(len(P.freqs)),
            "l2_policy": "inputs+outputs larger than L2 (126 MB) every step", "parallelism": "replicas"}


def sweep_measure(P, systems, maxit: int, precision: str, precond: str = "block_jacobi", tol: float = 1e-8,
                  network=None, fallback: bool = False, warmup: bool = True) -> dict:
    """Solves/s of one batched Krylov call: (frequency, port) systems driven to FP64 true relative
    residual <= tol, with the device assembly of E, B and the port terms (and, for the aux-space
    preconditioners, the aux space and its operator diagonals) inside the timed region.  One untimed
    run of the same arm on a two-system batch comes first (driver and allocator warm-up)."""
    import torch
    from emerge_b200.sweep import FrequencySweep
    if warmup:
        w = FrequencySweep(P)
        if network is not None:
            w.set_network(network)
        w.solve(systems[:2], tol=tol, maxit=maxit, precond=precond, precision=precision, fallback=fallback)
        del w
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sw = FrequencySweep(P)
    if network is not None:
        sw.set_network(network)
    res = sw.solve(systems, tol=tol, maxit=maxit, precond=precond, precision=precision, fallback=fallback)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    conv = int(((res.status == 0) & (res.relres <= tol)).sum())
    return {"precision": precision, "precond": precond, "method": "bicgstab", "systems": len(systems),
            "converged": conv, "seconds": dt, "solve_seconds": res.seconds, "solves_per_s": conv / dt,
            "iters_max": int(res.iters.max()), "iters_mean": float(res.iters.mean()),
            "relres_max": float(res.relres.max()), "maxit": maxit, "tol": tol, "fallback_systems": res.fallbacks}


def train_network(P, train_freqs, steps: int = 300) -> tuple:
    """Train the aux-space network on residual/correction pairs of the sweep's own solves at
    training frequencies (disjoint from the measured ones); returns (network, report dict)."""
    import torch
    from emerge_b200.auxspace import Network, make_pairs, train
    from emerge_b200.sweep import FrequencySweep
    sw = FrequencySweep(P)
    aux = sw.aux_space()
    t0 = time.perf_counter()
    pairs = make_pairs(sw, [(float(f), q) for f in train_freqs for q in range(len(P.ports))], snapshots=(4, 16, 48, 128))
    held = make_pairs(sw, [(float(0.5 * (train_freqs[0] + train_freqs[1])), 0)], snapshots=(16, 64))
    t_pairs = time.perf_counter() - t0
    net = Network(aux, seed=0)
    val = [(float(0.5 * (train_freqs[2] + train_freqs[3])), q) for q in range(len(P.ports))]
    rep = train(net, sw, pairs, heldout=held, steps=steps, batch=8, lr=2e-3, validate=val)
    torch.cuda.synchronize()
    return net, {"pairs": rep.pairs, "pair_seconds": t_pairs, "steps": rep.steps, "train_seconds": rep.seconds,
                 "validation_iters_aux_jacobi": rep.validation_iters_aux,
                 "validation_iters_learned": rep.validation_iters_learned, "accepted": rep.accepted,
                 "output_scale": rep.output_scale,
                 "validation_iters_by_output_scale": {str(k): v for k, v in rep.validation_by_scale.items()},
                 "loss_first": rep.loss_first, "loss_last": rep.loss_last,
                 "heldout_loss_aux_jacobi": rep.loss_jacobi_heldout, "heldout_loss_learned": rep.loss_learned_heldout,
                 "objective": "mean ||G za - e||^2 / ||e||^2 over (residual, correction) pairs"}


def batched_sweep_section(tol: float = 1e-8, maxit: int = 40000) -> dict:
    """Several meshes' sweeps in one batched Krylov call (``BatchSweep``) against the same meshes solved
    one ``FrequencySweep`` after another: 8 air-filled guides of uneven size (3 000-12 600 tets), two
    frequencies x two ports each, BiCGStab FP64 to ``tol`` with plain block Jacobi and with the aux-space
    correction; set-up (assembly, ports, aux space) and solve inside the timed regions."""
    import torch
    from emerge_b200 import problems
    from emerge_b200.batch import BatchSweep
    from emerge_b200.sweep import FrequencySweep
    rng = np.random.default_rng(5)
    Ps, systems = [], []
    for i in range(8):
        nx, ny, nz = int(rng.integers(8, 13)), int(rng.integers(4, 7)), int(rng.integers(12, 26))
        a = 22.86e-3 * rng.uniform(0.9, 1.1)
        Ps.append(problems.waveguide(nx=nx, ny=ny, nz=nz, a=a, seed=100 + i))
        fc = 299792458.0 / (2 * a)
        systems.append([(f, q) for f in (1.35 * fc, 1.75 * fc) for q in range(2)])
    tets = sum(P.mesh.n_tets for P in Ps)
    out = {"workload": "8 air-filled guides, 3 000-12 600 tets, 2 frequencies x 2 ports each, BiCGStab FP64 "
                       f"to {tol:g}", "meshes": len(Ps), "total_tets": int(tets), "systems": 4 * len(Ps)}
    for pc in ("block_jacobi", "aux"):
        BatchSweep(Ps[:2]).solve(systems[:2], tol=tol, maxit=50, precond=pc)    # driver / allocator warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bs = BatchSweep(Ps)
        rb = bs.solve(systems, tol=tol, maxit=maxit, precond=pc)
        torch.cuda.synchronize()
        t_b = time.perf_counter() - t0
        conv_b = sum(int(((r.status == 0) & (r.relres <= tol)).sum()) for r in rb)
        del bs
        gc.collect()
        t0 = time.perf_counter()
        conv_s, its_s = 0, []
        for P, sl in zip(Ps, systems):
            r = FrequencySweep(P).solve(sl, tol=tol, maxit=maxit, precond=pc)
            conv_s += int(((r.status == 0) & (r.relres <= tol)).sum())
            its_s.append(int(r.iters.max()))
        torch.cuda.synchronize()
        t_s = time.perf_counter() - t0
        out[pc] = {"batched": {"seconds": t_b, "converged": conv_b, "solves_per_s": conv_b / t_b,
                               "iters_max": int(max(int(r.iters.max()) for r in rb))},
                   "one_mesh_at_a_time": {"seconds": t_s, "converged": conv_s, "solves_per_s": conv_s / t_s,
                                          "iters_max_per_mesh": its_s}}
    return out


def precision_section(reps: int = 3) -> dict:
    """The precision workload: assembly of the full 1 497 600-tet substrate box (80x60x52 grid x 6), and
    on a downsized member (20x15x13 grid, 23 400 tets) the FP32-inner / FP64-refinement sweep against
    the FP64 sweep at two frequencies x two lumped ports (relative difference of the solutions per
    system; the FP64 solve itself is checked against the direct solve in the tests)."""
    import torch
    from emerge_b200 import problems
    from emerge_b200.assembly import CsrPlan, DeviceMesh
    from emerge_b200.sweep import FrequencySweep
    t0 = time.perf_counter()
    P = problems.substrate_box()
    t_mesh = time.perf_counter() - t0
    dev = torch.device("cuda", torch.cuda.current_device())
    dm = DeviceMesh(P.mesh, P.field, dev)
    plan = CsrPlan(dm)
    er = torch.from_numpy(np.ascontiguousarray(P.er)).to(dev)
    ur = torch.from_numpy(np.ascontiguousarray(P.ur)).to(dev)
    E, B = plan.assemble(er, ur)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        E, B = plan.assemble(er, ur, E, B)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    out = {"workload": "substrate box 16x12x10.4 mm, 80x60x52 hex grid x6 tets, eps_r 3.5-0.007j below grid plane 10, "
                       "PEC strip W/10 on the interface, lumped ports at both ends, order-2 ABC on the end faces",
           "n_tets": int(P.mesh.n_tets), "n_dof": int(P.field.n_field), "nnz": int(plan.nnz),
           "assembly_ms": ms, "assembly_tets_per_s": P.mesh.n_tets / (ms / 1e3), "host_mesh_seconds": t_mesh}
    del E, B, plan, dm, er, ur
    gc.collect()
    torch.cuda.empty_cache()
    Q = problems.substrate_box(20, 15, 13)
    sw = FrequencySweep(Q)
    systems = [(f, q) for f in (4.5e9, 8e9) for q in range(2)]
    r64 = sweep_measure(Q, systems, 40000, "fp64", "aux", tol=1e-8)
    rmx = sweep_measure(Q, systems, 40000, "mixed", "aux", tol=1e-8, fallback=True)
    a = sw.solve(systems, tol=1e-8, maxit=40000, precond="aux").x
    b = sw.solve(systems, tol=1e-8, maxit=40000, precond="aux", precision="mixed", fallback=True).x
    diff = (torch.linalg.vector_norm(a - b, dim=0) / torch.linalg.vector_norm(a, dim=0)).cpu().numpy()
    out["downsized"] = {"workload": "same family, 20x15x13 grid x6 (23 400 tets), 4.5 and 8 GHz x 2 ports to 1e-8",
                        "fp64_aux": r64, "mixed_aux_with_fallback": rmx,
                        "mixed_vs_fp64_rel_diff": [float(v) for v in diff]}
    return out


def batch_section(n_meshes: int = 64, seed: int = 7, reps: int = 3) -> dict:
    """Uneven meshes assembled in one launch: box meshes with seeded grid sizes giving 5 000-200 000
    tets each, per-tet eps' ~ U[1,12], tan d ~ U[0,5e-3], diagonal mu_r ~ U[1,2] on a seeded 10 % of tets
    (the reference has no batched form; each of its calls assembles one mesh)."""
    import torch
    from emerge_b200.batch import MeshBatch
    from emerge_b200.mesh import box_tet_mesh
    rng = np.random.default_rng(seed)
    meshes, ers, urs = [], [], []
    for i in range(n_meshes):
        target = rng.uniform(5000, 200000) / 6
        nx = max(2, int(round(target ** (1 / 3) * rng.uniform(0.7, 1.3))))
        ny = max(2, int(round((target / nx) ** 0.5 * rng.uniform(0.8, 1.2))))
        nz = max(2, int(round(target / (nx * ny))))
        a = 0.02 * rng.uniform(0.8, 1.25)
        nodes, tets = box_tet_mesh(nx, ny, nz, a, a * ny / nx, a * nz / nx, jitter=0.1, seed=1000 + i)
        meshes.append((nodes, tets))
        nt = tets.shape[1]
        d = rng.uniform(1, 12, nt) * (1 - 1j * rng.uniform(0, 5e-3, nt))
        er = np.zeros((3, 3, nt), np.complex128)
        ur = np.zeros((3, 3, nt), np.complex128)
        aniso = rng.random(nt) < 0.1
        for c in range(3):
            er[c, c] = d
            ur[c, c] = np.where(aniso, rng.uniform(1, 2, nt), 1.0)
        ers.append(er); urs.append(ur)
    sizes = [t.shape[1] for _, t in meshes]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b = MeshBatch(meshes)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    er = torch.from_numpy(np.concatenate(ers, axis=2)).cuda()
    ur = torch.from_numpy(np.concatenate(urs, axis=2)).cuda()
    del ers, urs
    b.assemble(er, ur)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        b.assemble(er, ur)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    out = {"workload": f"{n_meshes} box meshes, seeded grids giving {min(sizes)}-{max(sizes)} tets each, random "
                       "per-tet eps/mu, all assembled by one fused launch", "meshes": n_meshes,
           "total_tets": int(sum(sizes)), "nnz": int(b.plan.nnz), "ms_per_launch": ms,
           "tets_per_s": sum(sizes) / (ms * 1e-3), "setup_seconds_connectivity_plan": t_setup}
    del b, er, ur
    torch.cuda.empty_cache()
    return out


def configs_sweep_section(n_meshes: int = 16, tol: float = 1e-8) -> dict:
    """Configurations 3 and 4 as sweeps (opt-in, ``--configs-sweeps``; minutes of GPU time).

    Config 3: the first ``n_meshes`` of the 64 batched guides (``problems.batch_family``), 16 frequencies
    each, port 1 excited: the device LU sweep of every guide (``solve_direct``, adaptive windows, the
    symbolic set-up inside the timed region), against the batched aux-space Krylov solve of the same
    systems in one grouped launch (``BatchSweep``).  Config 4: the substrate family at 40 x 30 x 26 x 6 =
    187 200 tets, all 51 frequencies through the device LU, and the FP64 aux-space Krylov solve at the
    top 8 frequencies, with the relative difference of the two solutions per frequency."""
    import torch
    from emerge_b200 import problems
    from emerge_b200.batch import BatchSweep
    from emerge_b200.sweep import FrequencySweep
    out = {}
    Ps = problems.batch_family(64)[:n_meshes]
    systems = [[(float(f), 0) for f in P.freqs] for P in Ps]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lu_conv, lu_setup, lu_iters = 0, 0.0, 0
    for P, sl in zip(Ps, systems):
        ts = time.perf_counter()
        sw = FrequencySweep(P)
        sw.direct_solver()
        lu_setup += time.perf_counter() - ts
        rd = sw.solve_direct(sl, window=5, tol=tol, adaptive=True)
        lu_conv += int(((rd.status == 0) & (rd.relres <= tol)).sum())
        lu_iters = max(lu_iters, int(rd.iters.max()))
        del sw, rd
        gc.collect()
    torch.cuda.synchronize()
    t_lu = time.perf_counter() - t0
    torch.cuda.empty_cache()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bs = BatchSweep(Ps)
    rb = bs.solve(systems, tol=tol, maxit=6000, precond="aux")
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    conv_k = int(sum(((r.status == 0) & (r.relres <= tol)).sum() for r in rb))
    del bs, rb
    n_sys = sum(len(sl) for sl in systems)
    out["config3_batched_guides"] = {
        "workload": f"{n_meshes} of the 64 batched guides ({sum(P.mesh.n_tets for P in Ps)} tets, "
                    f"{min(P.mesh.n_tets for P in Ps)}-{max(P.mesh.n_tets for P in Ps)} each), 16 frequencies "
                    "over each guide's TE10-TE20 band, port 1 excited, FP64 relative residual 1e-8",
        "systems": n_sys,
        "device_lu": {"converged": lu_conv, "seconds": t_lu, "setup_seconds_in_it": lu_setup,
                      "iters_max": lu_iters, "solves_per_s": lu_conv / t_lu},
        "krylov_aux_batched": {"converged": conv_k, "seconds": t_batch, "solves_per_s": conv_k / t_batch}}
    gc.collect()
    torch.cuda.empty_cache()
    Q = problems.substrate_box(40, 30, 26)
    sw = FrequencySweep(Q)
    sys4 = [(float(f), 0) for f in Q.freqs]
    ts = time.perf_counter()
    sw.direct_solver()
    t_setup = time.perf_counter() - ts
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rd = sw.solve_direct(sys4, window=9, tol=tol, adaptive=True, precision="auto")
    torch.cuda.synchronize()
    t_d = time.perf_counter() - t0
    rk = sw.solve(sys4[-8:], tol=tol, maxit=30000, precond="aux")
    diff = []
    for j, (f, _) in enumerate(sys4[-8:]):
        if rk.status[j] == 0:
            xd = rd.x[:, len(sys4) - 8 + j]
            diff.append((f, float(torch.linalg.vector_norm(rk.x[:, j] - xd) / torch.linalg.vector_norm(xd))))
    out["config4_substrate_downsized"] = {
        "workload": "substrate box 40x30x26 hex grid x6 (187 200 tets), eps_r 3.5-0.007j below the interface, "
                    "PEC strip, lumped ports, order-2 ABC; all 51 frequencies 1-8 GHz, FP64 relative residual 1e-8",
        "device_lu": {"converged": int(((rd.status == 0) & (rd.relres <= tol)).sum()), "systems": len(sys4),
                      "seconds": t_d, "solves_per_s": int(((rd.status == 0) & (rd.relres <= tol)).sum()) / t_d,
                      "setup_seconds": t_setup, "iters_max": int(rd.iters.max()),
                      "relres_max": float(rd.relres.max()), "windows": len(rd.windows),
                      "precision": "auto (complex64 first, complex128 for the systems it leaves)",
                      "factorizations_c128": sum(1 for w in rd.windows
                                                 if w["precision"] == "c128" and w.get("factor_seconds", 0) > 0),
                      "c128_frequencies_max": max([w["factored"] for w in rd.windows
                                                   if w["precision"] == "c128" and "error" not in w],
                                                  default=None)},
        "aux_krylov_top8_freqs": {"converged": int((rk.status == 0).sum()), "seconds": rk.seconds,
                                  "iters_max": int(rk.iters.max())},
        "lu_vs_aux_rel_diff_per_freq": diff}
    return out


SWEEP_ARMS = ("plain_block_jacobi_fp64", "aux_jacobi_fp64", "aux_jacobi_mixed", "learned_fp64", "learned_mixed",
              "device_lu_c64_fp64_bicgstab")


def direct_measure(P, systems, window: int, tol: float = 1e-8, maxit: int = 400, sweep=None,
                   adaptive: bool = False) -> dict:
    """Solves/s of the device-LU sweep (``FrequencySweep.solve_direct``): per window of ``window``
    frequencies one complex64 multifrontal factorization at the middle frequency (K_f formed on the device)
    and FP64 BiCGStab preconditioned with it for every system of the window.  The timed region holds the
    factorizations and the solves; the per-mesh set-up (E/B assembly, nested-dissection ordering and front
    structure on the host, device allocation of the factor storage) is timed separately."""
    import torch
    from emerge_b200.sweep import FrequencySweep
    t0 = time.perf_counter()
    sw = sweep if sweep is not None else FrequencySweep(P)
    lu = sw.direct_solver()
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = sw.solve_direct(systems, window=window, tol=tol, maxit=maxit, adaptive=adaptive)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    conv = int(((res.status == 0) & (res.relres <= tol)).sum())
    fac = [w["factor_seconds"] for w in res.windows if w["factor_seconds"] > 0]
    out = {"precision": "complex64 LU factors and triangular solves inside FP64 BiCGStab (FP64 residual)",
           "precond": "device multifrontal LU of the window's middle frequency", "method": "bicgstab",
           "systems": len(systems), "window_frequencies": window, "adaptive_windows": adaptive,
           "converged": conv, "seconds": dt,
           "solves_per_s": conv / dt, "iters_max": int(res.iters.max()), "iters_mean": float(res.iters.mean()),
           "relres_max": float(res.relres.max()), "tol": tol, "maxit": maxit,
           "setup_seconds": t_setup, "setup_symbolic_seconds": lu.seconds_symbolic,
           "factor_seconds_mean": float(np.mean(fac)) if fac else None,
           "factor_tflops_c64": lu.flops / float(np.mean(fac)) / 1e12 if fac else None,
           "factor_flops": lu.flops, "factor_device_gb": lu.device_bytes / 1e9, "fronts": lu.n_fronts,
           "perturbed_pivots": int(max(w["perturbed"] for w in res.windows)),
           "windows": [{k: v for k, v in w.items()} for w in res.windows]}
    return out


def sweep_section(P_cavity, cavity_systems: int, cavity_maxit: int, arm_names=SWEEP_ARMS, lu_window: int = 5,
                  lu_windows: int = 2) -> dict:
    from emerge_b200 import problems
    wg = problems.waveguide()
    wg_sys = [(float(f), q) for f in np.linspace(8e9, 12e9, 16) for q in range(2)]
    net, trep = None, None
    if any(a.startswith("learned") for a in arm_names):
        net, trep = train_network(wg, np.linspace(8.125e9, 11.875e9, 9))
    spec = {
        "plain_block_jacobi_fp64": lambda: sweep_measure(wg, wg_sys, 40000, "fp64", "block_jacobi"),
        "aux_jacobi_fp64": lambda: sweep_measure(wg, wg_sys, 40000, "fp64", "aux"),
        "aux_jacobi_mixed": lambda: sweep_measure(wg, wg_sys, 40000, "mixed", "aux", fallback=True),
        "learned_fp64": lambda: sweep_measure(wg, wg_sys, 40000, "fp64", "learned", network=net, fallback=True),
        "learned_mixed": lambda: sweep_measure(wg, wg_sys, 40000, "mixed", "learned", network=net, fallback=True),
        "device_lu_c64_fp64_bicgstab": lambda: direct_measure(wg, wg_sys, window=4),
    }
    arms = {name: spec[name]() for name in SWEEP_ARMS if name in arm_names}
    plain = arms.get("plain_block_jacobi_fp64", {}).get("solves_per_s")
    auxj = arms.get("aux_jacobi_fp64", {}).get("solves_per_s")
    lfp = arms.get("learned_fp64", {}).get("solves_per_s")

    def ratio(a, b):
        return a / b if a and b else None
    out = {"waveguide_6000_tets": {
        "workload": "22.86x10.16x50 mm air guide, 10x5x20 hex grid x6 tets, TE10 ports, 16 frequencies 8-12 GHz "
                    "x 2 ports = 32 systems, FP64 true relative residual 1e-8",
        "arms": arms, "training": trep,
        # the network's own gain is learned against the aux-space Jacobi it starts from (the same
        # preconditioner with zero output weights); the aux-space structure's gain is aux against plain
        "network_gain_learned_vs_aux_jacobi_solves_per_s": ratio(lfp, auxj),
        "network_accepted": trep.get("accepted") if trep else None,
        "aux_jacobi_vs_plain_solves_per_s": ratio(auxj, plain),
        "device_lu_vs_plain_solves_per_s": ratio(arms.get("device_lu_c64_fp64_bicgstab", {}).get("solves_per_s"), plain)}}
    cav = {"workload": "the assembly workload (384 000 tets, 2 480 240 DOF, one TE10 port, PEC elsewhere): "
                       f"{'all' if lu_windows < 0 else lu_windows} windows of {lu_window} consecutive frequencies of the "
                       "101 (2-6 GHz) through the "
                       "device LU to FP64 relative residual 1e-8; block Jacobi and the aux-space correction with "
                       "bounded iterations (neither reaches 1e-8 on this cavity)"}
    if lu_windows != 0:
        if lu_windows < 0:            # every frequency of the sweep
            lu_sys = [(float(f), 0) for f in P_cavity.freqs]
        else:
            mid = len(P_cavity.freqs) // 2
            f0 = max(0, mid - (lu_window * lu_windows) // 2)
            lu_sys = [(float(f), 0) for f in P_cavity.freqs[f0:f0 + lu_window * lu_windows]]
        cav["device_lu_c64_fp64_bicgstab"] = direct_measure(P_cavity, lu_sys, window=lu_window,
                                                            adaptive=lu_windows < 0)
        import gc as _gc
        _gc.collect()
        import torch as _torch
        _torch.cuda.empty_cache()
    if cavity_systems > 0:
        cav_sys = [(float(f), 0) for f in P_cavity.freqs[:: max(1, len(P_cavity.freqs) // cavity_systems)][:cavity_systems]]
        cav["plain_block_jacobi_fp64"] = sweep_measure(P_cavity, cav_sys, cavity_maxit, "fp64", "block_jacobi")
        cav["aux_jacobi_fp64"] = sweep_measure(P_cavity, cav_sys, cavity_maxit, "fp64", "aux")
    out["cavity_384000_tets"] = cav
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--sweep-systems", type=int, default=4)
    ap.add_argument("--sweep-maxit", type=int, default=2000)
    ap.add_argument("--lu-window", type=int, default=9, help="frequencies per device-LU factorization on the cavity")
    ap.add_argument("--lu-windows", type=int, default=2,
                    help="cavity windows timed (0: skip the device-LU arm, -1: all 101 frequencies)")
    ap.add_argument("--sweep-arms", default=",".join(SWEEP_ARMS),
                    help="comma-separated waveguide sweep arms to measure (default: all)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--configs-sweeps", action="store_true",
                    help="also run configurations 3 and 4 as sweeps (several minutes of GPU time)")
    ap.add_argument("--grid", type=int, default=40, help="cavity hex grid size (40 = the 384 000-tet workload)")
    ap.add_argument("--variant", type=int, default=-1, help="assembly kernel variant (default: autotune)")
    args = ap.parse_args()
    ws, rank, local = dist_init(args.gpus)
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    from emerge_b200 import assembly, problems
    from emerge_b200._lib import Handle

    assert torch.cuda.is_available(), "bench.py needs a GPU"
    dev = torch.device("cuda", local if ws > 1 else 0)
    P = problems.cavity(n=args.grid)
    nt, N = P.mesh.n_tets, P.field.n_field
    dm = assembly.DeviceMesh(P.mesh, P.field, dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plan = assembly.CsrPlan(dm)
    torch.cuda.synchronize()
    t_plan = time.perf_counter() - t0
    nnz = plan.nnz
    er = torch.from_numpy(np.ascontiguousarray(P.er)).to(dev)
    ur = torch.from_numpy(np.ascontiguousarray(P.ur)).to(dev)
    E = torch.empty(nnz, dtype=torch.complex128, device=dev)
    B = torch.empty(nnz, dtype=torch.complex128, device=dev)
    stream = torch.cuda.current_stream(dev)

    if args.variant >= 0:
        plan.set_variant(args.variant)
        tuning = {"variant": args.variant, "ms": None}
    else:
        tuning = plan.tune(er, ur)
    tuned_info = plan.variant_info(int(tuning["variant"]))
    tuning = dict(tuning, **tuned_info)
    for _ in range(args.warmup):
        plan.assemble(er, ur, E, B)
    torch.cuda.synchronize()
    Handle.get(dev).raise_on_device_status("bench warm-up")

    # ---- device-resident timed region (inputs resident in HBM) ----
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        ev0.record(stream)
        for a, b in step_events:
            a.record(stream)
            plan.assemble(er, ur, E, B)
            b.record(stream)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(ws)
    total_ms = ev0.elapsed_time(ev1)
    step_ms = [a.elapsed_time(b) for a, b in step_events]
    ms_step = max_over_ranks(ws, total_ms / args.steps)
    value = ws * nt / (ms_step / 1e3)
    clocks = clk.summary()

    # ---- roofline of the assembly launch pair (invariants + row-owner assembly) ----
    hbm, peak_kind = peaks()
    alg_bytes_per_tet = 480 + 32.0 * nnz / nt
    achieved = nt * alg_bytes_per_tet / (float(np.mean(step_ms)) / 1e3) / 1e9

    # ---- end-to-end through the public API with host buffers ----
    from emerge_b200.assembly import tet_mass_stiffness_matrices
    host_in = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in
               (P.mesh.nodes, P.mesh.tets, P.mesh.tet_to_edge, P.mesh.edge_lengths, P.er, P.ur)]
    h2d = sum(t.numel() * t.element_size() for t in host_in)
    d2h = 2 * nnz * 16          # E and B values; the CSR pattern is downloaded once per plan
    P.field._emfem_cache = (("cuda:%d" % dev.index, id(P.mesh)), dm, plan)
    e2e_steps = max(2, min(args.steps, 4))
    # warm-up with the timed loop's own pattern (the previous results stay referenced while the
    # next call runs), so the plan's pinned result buffers exist before timing
    for _ in range(3):
        Eh, Bh = tet_mass_stiffness_matrices(P.field, host_in[4], host_in[5], device=dev)
    barrier(ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        dm.nodes.copy_(host_in[0], non_blocking=True)
        dm.tets.copy_(host_in[1], non_blocking=True)
        dm.tet_to_edge.copy_(host_in[2], non_blocking=True)
        dm.edge_lengths.copy_(host_in[3], non_blocking=True)
        Eh, Bh = tet_mass_stiffness_matrices(P.field, host_in[4], host_in[5], device=dev)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(ws, (time.perf_counter() - t0) / e2e_steps)
    e2e_value = ws * nt / e2e_s
    # release the drop-in's pinned result buffers (GBs of page-locked host memory) before the other
    # sections: right after such an allocation the driver's next set-up calls run much slower
    del Eh, Bh
    from emerge_b200.assembly import release_host_buffers
    release_host_buffers(P.field)
    import gc
    gc.collect()
    torch.cuda.synchronize()

    out = None
    if rank == 0:
        sweep = None
        if not args.no_sweep:
            sweep = sweep_section(P, args.sweep_systems, args.sweep_maxit,
                                  tuple(a for a in args.sweep_arms.split(",") if a), args.lu_window, args.lu_windows)
        batch = None if args.no_batch else batch_section()
        precision = None if args.no_precision else precision_section()
        batched_sweeps = None if args.no_batch else batched_sweep_section()
        cfg = configs_sweep_section() if args.configs_sweeps else None
        cb = None if args.no_cpu_baseline else cpu_baseline(P)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": workload_config(P),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": ASM_TRAFFIC_PER_TET * nt,
                         "traffic_note": "bytes per launch of assemble_chunk_kernel: dram read+write per tet from the "
                                         "ncu capture at 82 944 tets (profiles/assemble_chunk_kernel_cavity24.md) "
                                         "scaled by tets; the invariants kernel adds ~1.4 KB/tet",
                         "peak_kind": peak_kind,
                         "alg_bytes_per_tet": alg_bytes_per_tet,
                         "kernels": "tet_invariants_kernel+assemble_chunk_kernel"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "api": "emerge_b200.assembly.tet_mass_stiffness_matrices (host numpy in, SciPy CSR out)"},
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
            "plan_seconds": t_plan, "nnz": int(nnz), "autotune": tuning,
            "sweep": sweep,
            "batched_meshes": batch,
            "precision_workload": precision,
            "batched_sweeps": batched_sweeps,
            "configs_sweeps": cfg,
            "cpu_baseline": cb,
        }
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
