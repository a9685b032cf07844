"""Device S-parameter extraction (port-face interpolation + mode overlap) against the reference."""
import numpy as np
import pytest
import torch

import oracle
from oracle import sparams as osp
from emerge_b200 import problems
from emerge_b200.ports import k0_of
from emerge_b200.sweep import FrequencySweep, SolveResult, sparam_corrections

pytestmark = pytest.mark.gpu


def test_overlap_of_reference_solutions_matches_reference_S(cuda, golden):
    """Extraction alone: the reference's SuperLU solutions through the device kernel give the
    reference's raw S-matrix."""
    g = golden("config1")
    P = problems.waveguide()
    sw = FrequencySweep(P)
    f = float(g["f"])
    x = torch.from_numpy(np.ascontiguousarray(np.stack([g["x1"], g["x2"]], axis=1))).to(sw.device)
    res = SolveResult(x, np.zeros(2, int), np.zeros(2, int), np.zeros(2), [(f, 0), (f, 1)], 0.0)
    S = sw.sparams(res)[f]
    assert np.abs(S - g["S"]).max() <= 1e-12


def test_sweep_sparams_vs_direct_solve(cuda, golden):
    """Full device path (assembly, BiCGStab to 1e-12, extraction) vs the reference's S (<= 1e-6)."""
    g = golden("config1")
    P = problems.waveguide()
    sw = FrequencySweep(P)
    f = float(g["f"])
    res = sw.solve([(f, 0), (f, 1)], tol=1e-12, maxit=60000)
    assert (res.status == 0).all(), (res.status, res.iters, res.relres)
    S = sw.sparams(res)[f]
    assert np.abs(S - g["S"]).max() <= 1e-6
    assert abs(abs(S[1, 0]) - 1) < 0.01 and abs(S[0, 0]) < 0.01      # matched straight guide
    assert np.all(np.abs(sparam_corrections(S)) <= 1.0 + 1e-15)


def test_sparams_other_mesh_vs_oracle(cuda):
    P = problems.waveguide(nx=6, ny=3, nz=12, seed=5, shuffle_local=True)
    sw = FrequencySweep(P)
    f = 9e9
    res = sw.solve([(f, 0), (f, 1)], tol=1e-10, maxit=60000)
    x = res.x.cpu().numpy()
    S_dev = sw.sparams(res)[f]
    S_or = osp.sparams(P, {0: x[:, 0], 1: x[:, 1]}, k0_of(f), oracle.dunavant4())
    assert np.abs(S_dev - S_or).max() <= 1e-12


def test_lumped_port_sparams_match_oracle(cuda):
    """A guide with a TE10 port at z=0 and a lumped port on the z=l face: the device S (mode overlap
    and voltage lines) against the oracle's from the same device solutions."""
    from oracle import sparams as osp
    from emerge_b200.ports import LumpedPort
    P = problems.waveguide()
    a, b, l = P.dims
    P.ports = [P.ports[0], LumpedPort(2, P.ports[1].tri_ids, width=a, height=b, direction=(0.0, 1.0, 0.0))]
    sw = FrequencySweep(P)
    f = 10e9
    res = sw.solve([(f, 0), (f, 1)], tol=1e-11, maxit=20000, precond="aux")
    assert (res.status == 0).all()
    S = sw.sparams(res)[f]
    x = res.x.cpu().numpy()
    So = osp.sparams(P, {0: x[:, 0], 1: x[:, 1]}, k0_of(f), oracle.dunavant4())
    assert np.abs(S - So).max() <= 1e-9 * max(1.0, np.abs(So).max()), (S, So)
    assert np.isfinite(S).all()
