"""Frequency / mesh partition + result gather across 2 ranks (gloo on CPU, world size 2): the
round-robin and cost-balanced deals, and two CPU ranks solving real (small) guide systems dealt by
their cost (the solves by the oracle's SuperLU, since the ranks have no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from emerge_b200 import distributed


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, systems, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = distributed.run_partitioned(systems, lambda batch: [(f * 2.0, p, rank) for f, p in batch],
                                          world, rank, batch=3)
        out_q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_partition_covers_every_system_once():
    systems = [(float(f), p) for f in range(11) for p in range(2)]
    shares = [distributed.partition(systems, 3, r) for r in range(3)]
    idx = sorted(i for s in shares for i, _ in s)
    assert idx == list(range(len(systems)))
    with pytest.raises(ValueError):
        distributed.partition(systems, 2, 2)


def test_gather_detects_missing():
    with pytest.raises(RuntimeError):
        distributed.gather([(0, "a")], 2)


def test_two_rank_gloo_sweep_partition():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    systems = [(float(f), p) for f in range(7) for p in range(2)]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, systems, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, res in results:
        assert len(res) == len(systems)
        for i, (v, port_, solver_rank) in enumerate(res):
            assert v == systems[i][0] * 2.0 and port_ == systems[i][1]
            assert solver_rank == i % 2       # round-robin ownership


def test_cost_partition_balances_and_covers_everything():
    rng = np.random.default_rng(3)
    cost = [float(c) for c in rng.integers(1, 100, 37)]
    items = list(range(37))
    for world in (2, 3, 5):
        shares = [distributed.partition(items, world, r, cost) for r in range(world)]
        idx = sorted(i for s in shares for i, _ in s)
        assert idx == items
        loads = [sum(cost[i] for i, _ in s) for s in shares]
        assert max(loads) - min(loads) <= max(cost)            # greedy LPT bound
        for s in shares:
            assert [i for i, _ in s] == sorted(i for i, _ in s)


def _guide_solution(spec):
    """SuperLU solution of one small guide at one frequency, port 1 excited (oracle matrices)."""
    import scipy.sparse.linalg as spl
    import oracle
    from emerge_b200 import problems
    from emerge_b200.ports import k0_of
    nx, nz, f = spec
    P = problems.waveguide(nx=nx, ny=2, nz=nz, seed=nx * 100 + nz)
    fld = P.field
    E, B = oracle.tet_mass_stiffness_matrices(fld, P.er, P.ur)
    k0 = k0_of(f)
    Bm = fld.empty_tri_matrix()
    p0, p1 = P.ports
    Bm, b = oracle.assemble_robin_bc_excited(fld, Bm, p0.tri_ids, lambda x, y, z: p0.get_Uinc(x, y, z, k0),
                                             p0.get_gamma(k0), oracle.dunavant4())
    Bm = oracle.assemble_robin_bc(fld, Bm, p1.tri_ids, p1.get_gamma(k0))
    K = (E - B * k0 ** 2 + fld.generate_csr(Bm)).tocsc()
    ids = P.solve_ids
    x = spl.spsolve(K[ids][:, ids], b[ids])
    return float(np.linalg.norm(x)), len(ids)


_SPECS = [(3, 4, 9e9), (5, 8, 10e9), (4, 6, 11e9), (6, 10, 9.5e9), (3, 5, 10.5e9)]


def _cost(spec):
    nx, nz, _ = spec
    return float(nx * 2 * nz)          # proportional to the mesh's DOFs


def _solver_worker(rank, world, port, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = distributed.run_partitioned(_SPECS, lambda batch: [(_guide_solution(s), rank) for s in batch],
                                          world, rank, batch=2, cost=[_cost(s) for s in _SPECS])
        out_q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_solves_real_systems_by_cost():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_solver_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [_guide_solution(s) for s in _SPECS]
    owner = {i: r for r in range(2) for i, _ in distributed.partition(_SPECS, 2, r, [_cost(s) for s in _SPECS])}
    for rank, res in results:
        assert len(res) == len(_SPECS)
        for i, ((nrm, nfree), solver_rank) in enumerate(res):
            assert (nrm, nfree) == expect[i]               # the same SuperLU arithmetic on every rank
            assert solver_rank == owner[i]
