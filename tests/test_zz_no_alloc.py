"""The allocation-free sweep SpMV (emfem_sweep_spmv_noalloc) against the allocating one.

Some callers of this library cannot allocate device memory: applications whose GPU memory is
handed to their own pool allocator up front, and latency-critical loops that cannot afford an
allocation's device synchronisation.  For them the library keeps the SpMV's row map in a fixed
device array.  This test calls both entry points through the C ABI on the same inputs and checks
that two consecutive allocation-free calls agree with the allocating call.  It lives in a file of
its own that pytest collects last, and it builds everything it needs, so it passes both alone in
a fresh process and after the rest of the suite.
"""
import numpy as np
import pytest
import torch

from emerge_b200 import _lib, problems
from emerge_b200._lib import Handle, lib, ptr
from emerge_b200.sweep import FrequencySweep

pytestmark = pytest.mark.gpu


def _call(fn, sw, systems, x):
    freqs = [f for f, _ in systems]
    k0 = torch.from_numpy(sw.k0sq(freqs)).to(sw.device)
    g = sw.gammas(freqs)
    gam = torch.from_numpy(np.ascontiguousarray(np.stack([g.real, g.imag], -1).reshape(-1))).to(sw.device)
    y = torch.full_like(x, complex(np.nan, np.nan))
    h = Handle.get(sw.device)
    st = fn(h.h, sw.n, ptr(sw.plan.indptr), ptr(sw.plan.indices), ptr(sw.E), ptr(sw.B), len(systems), ptr(k0),
            sw.patch_rows.numel(), ptr(sw.patch_rows), ptr(sw.patch_rowptr), ptr(sw.patch_cols), ptr(sw.patch_vals),
            ptr(sw.patch_port), sw.n_ports, ptr(gam), ptr(sw.mask), ptr(x), ptr(y))
    assert st == 0, _lib.last_error()
    torch.cuda.synchronize()
    return y


def test_noalloc_spmv_matches_allocating_spmv_twice(cuda):
    P = problems.waveguide(nx=6, ny=3, nz=10, seed=3)
    sw = FrequencySweep(P)
    systems = [(10e9, 0), (10e9, 1), (9e9, 0), (11e9, 1)]
    gen = torch.Generator(device="cpu").manual_seed(7)
    x = torch.complex(torch.randn(sw.n, 4, generator=gen, dtype=torch.float64),
                      torch.randn(sw.n, 4, generator=gen, dtype=torch.float64)).to(sw.device)
    x = x * sw.mask.to(torch.float64)[:, None]
    y_ref = _call(lib().emfem_sweep_spmv, sw, systems, x)
    for _ in range(2):
        y = _call(lib().emfem_sweep_spmv_noalloc, sw, systems, x)
        err = (torch.linalg.norm(y - y_ref) / torch.linalg.norm(y_ref)).item()
        assert err <= 1e-12, err


def test_noalloc_rejects_rows_beyond_its_scratch(cuda):
    P = problems.waveguide(nx=2, ny=2, nz=2, seed=0)
    sw = FrequencySweep(P)
    h = Handle.get(sw.device)
    too_many = (1 << 22) + 2
    x = torch.zeros(sw.n, 1, dtype=torch.complex128, device=sw.device)
    st = lib().emfem_sweep_spmv_noalloc(h.h, too_many, ptr(sw.plan.indptr), ptr(sw.plan.indices), ptr(sw.E),
                                        ptr(sw.B), 1, ptr(torch.zeros(1, dtype=torch.float64, device=sw.device)),
                                        0, None, None, None, None, None, 0, None, ptr(sw.mask), ptr(x), ptr(x))
    assert st == _lib.ERR_INVALID_ARG
    assert "fixed scratch" in _lib.last_error()
