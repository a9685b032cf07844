"""Host logic of FrequencySweep.solve_direct's precision policy (complex64 first, complex128 for the
systems it leaves; complex64 results standing when the complex128 workspace does not fit), run with a
stand-in sweep and LU on the CPU: the stand-in converges a system when the LU is complex128 or the
frequency is at least 2 GHz, as the substrate family does on the device."""
import numpy as np
import torch

from emerge_b200.sweep import FrequencySweep, SolveResult


class _LU:
    def __init__(self, c128_fits=True):
        self.precision = "c64"
        self.c128_fits = c128_fits
        self.n_perturbed = 0
        self.factored = []

    def set_precision(self, p):
        if p == "c128" and not self.c128_fits:
            raise RuntimeError("emfem_mf_set_precision: cudaMalloc failed")
        self.precision = p
        return self

    def factor(self, f):
        self.factored.append((f, self.precision))
        return self


class _Sweep:
    n = 4
    device = torch.device("cpu")

    def __init__(self, lu):
        self._lu = lu

    def direct_solver(self):
        return self._lu

    def solve_lu(self, systems, lu, tol=1e-8, maxit=500):
        k = len(systems)
        ok = np.array([lu.precision == "c128" or f >= 2e9 for f, _ in systems])
        x = torch.zeros((self.n, k), dtype=torch.complex128)
        for j, (f, _) in enumerate(systems):
            x[:, j] = f / 1e9 + (1j if lu.precision == "c128" else 0)
        return SolveResult(x, np.where(ok, 0, 1), np.where(ok, 3, maxit), np.where(ok, 1e-10, 1.0), list(systems), 0.0)


def _run(lu, precision="auto"):
    systems = [(f, 0) for f in (1e9, 1.5e9, 2e9, 3e9, 5e9, 8e9)]
    return FrequencySweep.solve_direct(_Sweep(lu), systems, window=2, tol=1e-8, precision=precision, probe_maxit=60)


def test_auto_solves_low_frequencies_again_in_complex128():
    lu = _LU()
    r = _run(lu)
    assert (r.status == 0).all()
    # windows of two frequencies, each factored at its second: the 1-1.5 GHz window fails in complex64 and
    # is refactored in complex128; that window converged quickly, so the next ones go back to complex64
    assert lu.factored == [(1.5e9, "c64"), (1.5e9, "c128"), (3e9, "c64"), (8e9, "c64")]
    x = r.x.numpy()
    assert np.all(x[:, :2].imag == 1) and np.all(x[:, 2:].imag == 0)
    assert all(w["precision"] in ("c64", "c128") for w in r.windows)


def test_auto_keeps_complex64_results_when_complex128_does_not_fit():
    lu = _LU(c128_fits=False)
    r = _run(lu)
    assert list(r.status[:2]) == [1, 1] and (r.status[2:] == 0).all()
    errs = [w for w in r.windows if "error" in w]
    assert len(errs) == 1                       # one failed switch, then the sweep stays complex64
    assert {p for _, p in lu.factored} == {"c64"}


def test_fixed_precisions_never_switch():
    for p in ("c64", "c128"):
        lu = _LU()
        r = _run(lu, precision=p)
        assert {q for _, q in lu.factored} == {p}
        assert (r.status == 0).all() == (p == "c128")
