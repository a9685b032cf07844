"""γ(k0) of the non-excited Robin boundaries against the reference's own get_gamma
(tests/golden/robin_gamma.npz, written by tests/golden/make_golden.py)."""
import numpy as np
import pytest

from emerge_b200.boundaries import ABC_O2_COEFFS, AbsorbingBoundary, SurfaceImpedance


def test_absorbing_boundary_gamma(golden):
    g = golden("robin_gamma")
    abc = AbsorbingBoundary(np.arange(3))
    got = np.array([abc.get_gamma(k) for k in g["k0"]])
    assert np.abs(got - g["abc1"]).max() <= 1e-14 * np.abs(g["abc1"]).max()
    for t in "ABCDE":       # the order-2 coefficient table, applied as the reference does
        got2 = np.array([1j * k * ABC_O2_COEFFS[t][0] for k in g["k0"]])
        assert np.abs(got2 - g["abc2_" + t]).max() <= 1e-14 * np.abs(g["abc2_" + t]).max()
    with pytest.raises(NotImplementedError):
        AbsorbingBoundary(np.arange(3), order=2)


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
