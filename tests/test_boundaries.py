"""γ(k0) of the non-excited Robin boundaries against the reference's own get_gamma
(tests/golden/robin_gamma.npz, written by tests/golden/make_golden.py)."""
import numpy as np
import pytest

from emerge_b200.boundaries import ABC_O2_COEFFS, AbsorbingBoundary, SurfaceImpedance


def test_absorbing_boundary_gamma(golden):
    g = golden("robin_gamma")
    abc = AbsorbingBoundary(np.arange(3), order=1)
    got = np.array([abc.get_gamma(k) for k in g["k0"]])
    assert np.abs(got - g["abc1"]).max() <= 1e-14 * np.abs(g["abc1"]).max()
    assert abc.get_gamma2(100.0) == 0.0
    for t in "ABCDE":       # order 2 (the reference's default): γ = j k0 c0, correction j c2 / k0
        abc2 = AbsorbingBoundary(np.arange(3), order=2, abctype=t)
        got2 = np.array([abc2.get_gamma(k) for k in g["k0"]])
        assert np.abs(got2 - g["abc2_" + t]).max() <= 1e-14 * np.abs(g["abc2_" + t]).max()
        assert abc2.get_gamma2(250.0) == 1j * ABC_O2_COEFFS[t][1] / 250.0
    assert AbsorbingBoundary(np.arange(3)).order == 2
    with pytest.raises(ValueError):
        AbsorbingBoundary(np.arange(3), order=3)


def test_abc2_oracle_matches_reference(golden):
    """The second-order ABC correction oracle reproduces the reference's abc_order_2_matrix."""
    from oracle import abc2
    from emerge_b200.mesh import TetMesh
    from emerge_b200.nedelec2 import Nedelec2
    g = golden("abc2")
    d = golden("element_small")
    f = Nedelec2(TetMesh(d["nodes"], d["tets"]))
    M = abc2.abc_order_2_matrix(f, g["tri_ids"], complex(g["cf"])).reshape(-1, 64)[g["tri_ids"]]
    assert np.abs(M - g["blocks"]).max() <= 1e-13 * np.abs(g["blocks"]).max()


@pytest.mark.parametrize("i", range(4))
def test_surface_impedance_gamma(golden, i):
    g = golden("robin_gamma")
    sigma, thick, sr, mur, er = g[f"surf{i}_params"]
    si = SurfaceImpedance(np.arange(3), sigma=sigma, mur=mur, epsr=er, thickness=None if thick < 0 else thick,
                          roughness=sr)
    got = np.array([si.get_gamma(k) for k in g["k0"]])
    ref = g[f"surf{i}"]
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_surface_impedance_function_gamma(golden):
    g = golden("robin_gamma")
    si = SurfaceImpedance(np.arange(3), impedance_function=lambda f: (0.02 + 1e-12 * f) + 1j * (0.01 + 3e-12 * f))
    got = np.array([si.get_gamma(k) for k in g["k0"]])
    assert np.abs(got - g["surf_fn"]).max() <= 1e-12 * np.abs(g["surf_fn"]).max()
    with pytest.raises(ValueError):
        SurfaceImpedance(np.arange(3))


@pytest.mark.parametrize("i,zp,pw", [(0, 50.0, 1.0), (1, 75.0, 0.5)])
def test_lumped_port_gamma_and_uinc(golden, i, zp, pw):
    from emerge_b200.ports import LumpedPort
    g = golden("robin_gamma")
    lp = LumpedPort(1, np.arange(3), width=2e-3, height=3e-3, direction=(0.6, 0.0, 0.8), power=pw, Z0=zp)
    got = np.array([lp.get_gamma(k) for k in g["k0"]])
    assert np.abs(got - g[f"lumped{i}_gamma"]).max() <= 1e-13 * np.abs(got).max()
    xs, ys, zs = np.array([1e-3, 2e-3]), np.array([0.5e-3, 0.0]), np.array([0.0, 1e-3])
    u = np.array([lp.get_Uinc(xs, ys, zs, k) for k in g["k0"]])
    ref = g[f"lumped{i}_uinc"]
    assert np.abs(u - ref).max() <= 1e-13 * np.abs(ref).max()


def test_voltage_line_rule_matches_reference(golden):
    """The lumped-port line integral: the reference's composite 3-point Gauss rule on equally spaced
    samples (coord.py:24-61) equals per-sample Simpson weights."""
    from oracle.sparams import simpson_line_weights
    g = golden("robin_gamma")
    got = simpson_line_weights(21) @ g["line_samples"]
    assert abs(got - complex(g["line_gauss3"])) <= 1e-14 * abs(complex(g["line_gauss3"]))
