"""Several meshes' sweeps in one batched Krylov call (``BatchSweep`` over
``emfem_krylov_solve_grouped``) against each mesh solved on its own."""
import numpy as np
import pytest
import torch

from emerge_b200 import problems
from emerge_b200._lib import EmfemError
from emerge_b200.batch import BatchSweep
from emerge_b200.boundaries import AbsorbingBoundary
from emerge_b200.sweep import FrequencySweep

pytestmark = pytest.mark.gpu


def _mixed_problems():
    P0 = problems.waveguide(nx=4, ny=2, nz=8, seed=1)
    P1 = problems.waveguide()
    P2 = problems.waveguide(nx=6, ny=3, nz=12, seed=2)
    # an absorbing boundary in place of P2's second port: a Robin term next to the ports
    P2.robin = [AbsorbingBoundary(P2.ports[1].tri_ids, order=2)]
    P2.ports = P2.ports[:1]
    return [P0, P1, P2]


def test_grouped_sweep_matches_separate_sweeps(cuda):
    Ps = _mixed_problems()
    bs = BatchSweep(Ps)
    systems = [[(9e9, 0), (9e9, 1), (11e9, 0)],
               [(10e9, 0), (10e9, 1), (8.5e9, 1)],
               [(12e9, 0), (8e9, 0), (10e9, 0)]]
    res = bs.solve(systems, tol=1e-11, maxit=60000)
    for g, P in enumerate(Ps):
        r = res[g]
        assert (r.status == 0).all(), (g, r.status, r.iters, r.relres)
        assert (r.relres <= 1e-11).all()
        ref = FrequencySweep(P).solve(systems[g], tol=1e-11, maxit=60000)
        assert (ref.status == 0).all()
        err = (torch.linalg.vector_norm(r.x - ref.x, dim=0) / torch.linalg.vector_norm(ref.x, dim=0)).cpu().numpy()
        assert err.max() <= 1e-8, (g, err)
        S, Sr = bs.sparams(g, r), FrequencySweep(P).sparams(ref)
        for f in S:
            assert np.nanmax(np.abs(S[f] - Sr[f])) <= 1e-8
        # independence of the groups: the same mesh batched alone has the same padded rows and block
        # sums, so it gives bit-identical solutions and iteration counts (against FrequencySweep the
        # counts differ by rounding only, which BiCGStab's stagnation phases can stretch)
        alone = BatchSweep([P]).solve([systems[g]], tol=1e-11, maxit=60000)[0]
        assert torch.equal(alone.x, r.x) and np.array_equal(alone.iters, r.iters), (alone.iters, r.iters)


def test_grouped_layout_is_validated(cuda):
    """A group that does not start on a 256-pair boundary is refused before any launch."""
    Ps = _mixed_problems()[:2]
    bs = BatchSweep(Ps)
    bad = bs.pair_group.clone()
    bad[bs.hoff[1] - 1] = 1                     # group 1 would start one pair early
    bs.pair_group = bad
    with pytest.raises(EmfemError):
        bs.solve([[(9e9, 0)], [(10e9, 0)]], tol=1e-8, maxit=10)


def test_grouped_aux_sweep_matches_separate_aux_sweeps(cuda):
    """precond="aux" over a batch: the union's auxiliary nodal space moved onto the grouped rows, its
    diagonals per system from each aux node's own mesh and frequency."""
    Ps = _mixed_problems()
    bs = BatchSweep(Ps)
    systems = [[(9e9, 0), (9e9, 1), (11e9, 0)],
               [(10e9, 0), (10e9, 1), (8.5e9, 1)],
               [(12e9, 0), (8e9, 0), (10e9, 0)]]
    res = bs.solve(systems, tol=1e-11, maxit=20000, precond="aux")
    for g, P in enumerate(Ps):
        r = res[g]
        assert (r.status == 0).all(), (g, r.status, r.iters, r.relres)
        ref = FrequencySweep(P).solve(systems[g], tol=1e-11, maxit=20000, precond="aux")
        assert (ref.status == 0).all()
        err = (torch.linalg.vector_norm(r.x - ref.x, dim=0) / torch.linalg.vector_norm(ref.x, dim=0)).cpu().numpy()
        assert err.max() <= 1e-8, (g, err)
        # the aux correction still cuts the iterations by an order of magnitude, as for one mesh
        assert r.iters.max() <= 3 * ref.iters.max() + 50, (r.iters, ref.iters)
        alone = BatchSweep([P]).solve([systems[g]], tol=1e-11, maxit=20000, precond="aux")[0]
        assert torch.equal(alone.x, r.x) and np.array_equal(alone.iters, r.iters), (alone.iters, r.iters)


def test_grouped_learned_sweep_matches_separate_learned_sweeps(cuda):
    """precond="learned" over a batch: one network (weights per aux-node type) on the union's aux space."""
    from emerge_b200.auxspace import Network
    Ps = _mixed_problems()
    bs = BatchSweep(Ps)
    net = Network(bs.aux_space(), seed=4, init="random")
    net.params.mul_(0.5)                         # a mild random correction that still converges
    bs.set_network(net)
    systems = [[(9e9, 0), (11e9, 0)], [(10e9, 0), (10e9, 1)], [(12e9, 0), (8e9, 0)]]
    res = bs.solve(systems, tol=1e-11, maxit=20000, precond="learned")
    for g, P in enumerate(Ps):
        r = res[g]
        assert (r.status == 0).all(), (g, r.status, r.iters, r.relres)
        sw = FrequencySweep(P)
        sw.set_network(Network(sw.aux_space(), params=net.params))
        ref = sw.solve(systems[g], tol=1e-11, maxit=20000, precond="learned")
        assert (ref.status == 0).all()
        err = (torch.linalg.vector_norm(r.x - ref.x, dim=0) / torch.linalg.vector_norm(ref.x, dim=0)).cpu().numpy()
        assert err.max() <= 1e-8, (g, err)


def test_grouped_mixed_precision_sweep_reaches_fp64_residual(cuda):
    """FP32 inner solves in FP64 refinement over a batch: every system of every mesh reaches the FP64
    true residual, each mesh's solutions as close to its own mixed-precision sweep as the tolerance allows,
    and each mesh batched alone gives the same bits."""
    Ps = _mixed_problems()
    bs = BatchSweep(Ps)
    systems = [[(9e9, 0), (11e9, 0)], [(10e9, 0), (10e9, 1)], [(12e9, 0), (8e9, 0)]]
    res = bs.solve(systems, tol=1e-8, maxit=20000, precond="aux", precision="mixed")
    for g, P in enumerate(Ps):
        r = res[g]
        assert (r.status == 0).all() and (r.relres <= 1e-8).all(), (g, r.status, r.iters, r.relres)
        ref = FrequencySweep(P).solve(systems[g], tol=1e-8, maxit=20000, precond="aux", precision="mixed")
        err = (torch.linalg.vector_norm(r.x - ref.x, dim=0) / torch.linalg.vector_norm(ref.x, dim=0)).cpu().numpy()
        assert err.max() <= 1e-5, (g, err)
        alone = BatchSweep([P]).solve([systems[g]], tol=1e-8, maxit=20000, precond="aux", precision="mixed")[0]
        assert torch.equal(alone.x, r.x), g
