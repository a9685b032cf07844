"""ctypes binding of ``libemfem.so`` (the C ABI declared in ``include/emfem.h``).

There is no fallback: if the library is missing or a call fails, an :class:`EmfemError` is raised.
Device buffers are torch tensors; their ``data_ptr()`` is passed straight through.
"""
from __future__ import annotations

import ctypes
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libemfem.so")

EMFEM_OK = 0
ERR_INVALID_ARG = -1
ERR_CUDA = -2
ERR_DEVICE_CHECK = -3
ERR_WORKSPACE = -4
ERR_NOT_CONVERGED = -5

DEV_BAD_INDEX = 1
DEV_DEGENERATE = 2
DEV_NONFINITE = 4
DEV_CAPACITY = 8
DEV_BREAKDOWN = 16


class EmfemError(RuntimeError):
    def __init__(self, msg: str, status: int):
        super().__init__(msg)
        self.status = status


_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int
_dbl = ctypes.c_double
_i32p = ctypes.POINTER(ctypes.c_int)
_dblp = ctypes.POINTER(ctypes.c_double)

_SIGS = {
    "emfem_version": ([], _i32),
    "emfem_last_error": ([ctypes.c_char_p, ctypes.c_size_t], _i32),
    "emfem_create": ([ctypes.POINTER(_vp), _i32, _vp], _i32),
    "emfem_set_stream": ([_vp, _vp], _i32),
    "emfem_destroy": ([_vp], _i32),
    "emfem_device_status": ([_vp, _i32p], _i32),
    "emfem_ned2_tet_matrices": ([_vp, _i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _i32),
    "emfem_ned2_coo_indices": ([_vp, _i64, _vp, _vp, _vp], _i32),
    "emfem_mesh_check": ([_vp, _i64, _i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp], _i32),
    "emfem_plan_create": ([_vp, _i64, _i64, _i64, _vp, ctypes.POINTER(_vp)], _i32),
    "emfem_plan_info": ([_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64)], _i32),
    "emfem_plan_destroy": ([_vp], _i32),
    "emfem_plan_export_csr": ([_vp, _vp, _vp], _i32),
    "emfem_plan_assemble": ([_vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _i32),
    "emfem_plan_find_slots": ([_vp, _i64, _vp, _vp, _vp], _i32),
    "emfem_plan_variants": ([_vp, _i32p, _i32p], _i32),
    "emfem_plan_set_variant": ([_vp, _i32], _i32),
    "emfem_plan_variant_info": ([_vp, _i32, _i32p, _i32p, _i32p], _i32),
    "emfem_ned2_tri_robin": ([_vp, _i64, _vp, _i64, _vp, _dbl, _dbl, _vp, _vp, _i32, _vp, _vp], _i32),
    "emfem_segmented_gather_sum": ([_vp, _i64, _vp, _vp, _vp, _vp], _i32),
    "emfem_sweep_combine": ([_vp, _i64, _vp, _vp, _dbl, _i64, _vp, _vp, _dbl, _dbl, _vp], _i32),
    "emfem_csr_drop_zeros_workspace": ([_i64, ctypes.POINTER(ctypes.c_size_t)], _i32),
    "emfem_csr_count_nonzero": ([_vp, _i64, _vp, _vp, _vp, _vp, ctypes.c_size_t, ctypes.POINTER(_i64)], _i32),
    "emfem_csr_compact_nonzero": ([_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp], _i32),
    "emfem_krylov_workspace_size": ([_i64, _i64, _i32, _i32, ctypes.POINTER(ctypes.c_size_t)], _i32),
    "emfem_krylov_solve": ([_vp, _i32, _i64, _i64, _vp, _vp, _vp, _vp, _i32, _dblp,
                          _i64, _vp, _vp, _vp, _vp, _vp, _i32, _dblp, _vp, _vp, _vp,
                          _dbl, _i32, _i32, _i32, _vp, ctypes.c_size_t, _i32p, _i32p, _dblp, _vp], _i32),
    "emfem_sweep_spmv": ([_vp, _i64, _vp, _vp, _vp, _vp, _i32, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _i32, _vp,
                          _vp, _vp, _vp], _i32),
    "emfem_port_overlap": ([_vp, _i64, _vp, _i64, _vp, _vp, _i64, _i64, _vp, _vp, _vp, _i32, _vp, _vp, _i32, _vp,
                            _vp, _vp, _vp], _i32),
    "emfem_mesh_connect_create": ([_vp, _i64, _i64, _vp, ctypes.POINTER(_vp)], _i32),
    "emfem_mesh_connect_info": ([_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64)], _i32),
    "emfem_mesh_connect_export": ([_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _i32),
    "emfem_mesh_connect_destroy": ([_vp], _i32),
    "emfem_aux_create": ([_vp, _i64, _i64, _i64, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)], _i32),
    "emfem_aux_info": ([_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)], _i32),
    "emfem_aux_export": ([_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _i32),
    "emfem_aux_set_operator": ([_vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _i32, _vp, _vp, _vp],
                               _i32),
    "emfem_aux_reserve": ([_vp, _i32], _i32),
    "emfem_aux_set_network": ([_vp, _vp], _i32),
    "emfem_aux_destroy": ([_vp], _i32),
    "emfem_aux_dinv": ([_vp, _i32, _vp, _vp, _vp], _i32),
    "emfem_aux_restrict": ([_vp, _i32, _vp, _vp, _vp], _i32),
    "emfem_aux_prolong": ([_vp, _i32, _vp, _vp, _vp, _i32], _i32),
    "emfem_mpnn_nparams": ([], _i32),
    "emfem_mpnn_workspace_floats": ([_vp, _i32, ctypes.POINTER(_i64), ctypes.POINTER(_i64)], _i32),
    "emfem_mpnn_forward": ([_vp, _i32, _vp, _vp, _vp, _vp], _i32),
    "emfem_mpnn_infer": ([_vp, _i32, _vp, _vp, _vp, _vp], _i32),
    "emfem_mpnn_backward": ([_vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp], _i32),
    "emfem_adam_step": ([_vp, _i64, _vp, _vp, _vp, _vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                         ctypes.c_float, ctypes.c_float, _i32], _i32),
    "emfem_ned2_tri_abc2": ([_vp, _i64, _vp, _i64, _vp, _dbl, _dbl, _vp], _i32),
    "emfem_ned2_bma_tri_matrices": ([_vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _dbl, _vp, _vp], _i32),
    "emfem_ned2_tri_field": ([_vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _i32, _vp, _i32, _dbl, _dbl, _vp, _vp], _i32),
    "emfem_krylov_workspace_size_grouped": ([_i64, _i64, _i32, _i32, _i32, ctypes.POINTER(ctypes.c_size_t)], _i32),
    "emfem_krylov_solve_grouped": ([_vp, _i32, _i64, _i64, _vp, _vp, _vp, _vp, _i32, _vp, _i32, _dblp,
                                    _i64, _vp, _vp, _vp, _vp, _vp, _i32, _dblp, _vp, _vp, _vp,
                                    _dbl, _i32, _i32, _i32, _vp, ctypes.c_size_t, _i32p, _i32p, _dblp, _vp], _i32),
    "emfem_aux_set_rows": ([_vp, _i64, _vp, _i32, _vp], _i32),
    "emfem_point_field_dot": ([_vp, _i64, _vp, _i64, _vp, _vp, _i64, _i64, _vp, _vp, _vp, _i32, _vp, _vp], _i32),
    "emfem_mf_create": ([_vp, _i64, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)], _i32),
    "emfem_mf_build_lists": ([_vp, _i64, _vp, _vp], _i32),
    "emfem_mf_info": ([_vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_double), _i32p], _i32),
    "emfem_mf_factor": ([_vp, _vp, _i32p], _i32),
    "emfem_mf_set_precision": ([_vp, _i32], _i32),
    "emfem_mf_reserve": ([_vp, _i32], _i32),
    "emfem_mf_solve": ([_vp, _i32, _vp, _vp], _i32),
    "emfem_mf_destroy": ([_vp], _i32),
    "emfem_krylov_solve_lu": ([_vp, _i64, _i64, _vp, _vp, _vp, _vp, _i32, _dblp, _i64, _vp, _vp, _vp, _vp, _vp, _i32,
                               _dblp, _vp, _vp, _vp, _dbl, _i32, _vp, _vp, ctypes.c_size_t, _i32p, _i32p, _dblp], _i32),
    "emfem_sweep_spmv_noalloc": ([_vp, _i64, _vp, _vp, _vp, _vp, _i32, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _i32,
                                  _vp, _vp, _vp, _vp], _i32),
}

_lib = None
_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise EmfemError(f"{LIB_PATH} is not built; run `python -m emerge_b200.build`", ERR_INVALID_ARG)
                L = ctypes.CDLL(LIB_PATH)
                for name, (args, res) in _SIGS.items():
                    fn = getattr(L, name)
                    fn.argtypes = args
                    fn.restype = res
                _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().emfem_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int, what: str = "") -> None:
    if status != EMFEM_OK:
        raise EmfemError(f"{what}: {last_error()} (status {status})", status)


def ptr(t) -> ctypes.c_void_p | None:
    if t is None:
        return None
    if isinstance(t, torch.Tensor):
        if not t.is_cuda:
            raise EmfemError("expected a CUDA tensor", ERR_INVALID_ARG)
        if not t.is_contiguous():
            raise EmfemError("expected a contiguous tensor", ERR_INVALID_ARG)
        return ctypes.c_void_p(t.data_ptr())
    return ctypes.c_void_p(int(t))


class Handle:
    """One ``emfem_handle`` per CUDA device; every call runs on torch's current stream."""

    _handles: dict[int, "Handle"] = {}

    def __init__(self, device: int):
        self.device = device
        h = _vp()
        with torch.cuda.device(device):
            check(lib().emfem_create(ctypes.byref(h), device, None), "emfem_create")
        self.h = h

    @classmethod
    def get(cls, device: int | torch.device | None = None) -> "Handle":
        if device is None:
            device = torch.cuda.current_device()
        if isinstance(device, torch.device):
            device = device.index if device.index is not None else torch.cuda.current_device()
        if device not in cls._handles:
            cls._handles[device] = Handle(device)
        hd = cls._handles[device]
        stream = torch.cuda.current_stream(device).cuda_stream
        lib().emfem_set_stream(hd.h, ctypes.c_void_p(stream))
        return hd

    def device_status(self) -> int:
        st = ctypes.c_int(0)
        check(lib().emfem_device_status(self.h, ctypes.byref(st)), "emfem_device_status")
        return st.value

    def raise_on_device_status(self, what: str) -> None:
        st = self.device_status()
        if st:
            names = [n for b, n in ((DEV_BAD_INDEX, "index out of range / inconsistent mesh"),
                                    (DEV_DEGENERATE, "degenerate element"),
                                    (DEV_NONFINITE, "non-finite input"),
                                    (DEV_CAPACITY, "per-entity capacity exceeded"),
                                    (DEV_BREAKDOWN, "breakdown")) if st & b]
            raise EmfemError(f"{what}: device check failed: {', '.join(names)} (bits {st})", ERR_DEVICE_CHECK)
