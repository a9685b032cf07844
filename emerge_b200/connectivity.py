"""Mesh connectivity on the GPU (``emfem_mesh_connect_*``), in ``Mesh3D`` conventions.

Replaces the Python-loop connectivity of ``Mesh3D._pre_update`` (``src/emerge/_emerge/mesh3d.py:385-497``)
for the arrays the FEM hot path reads: ``edges``, ``tris``, ``tet_to_edge``, ``tet_to_tri``,
``tri_to_edge``, ``tri_to_tet`` and ``edge_lengths``.  Ids are the reference's (lexicographic order
of the sorted node tuples), so a :class:`DeviceTetMesh` can stand in for a ``Mesh3D`` / ``TetMesh``
wherever those arrays are used, e.g. ``DeviceMesh(DeviceTetMesh(nodes, tets))``.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import Handle, check, lib, ptr

__all__ = ["DeviceTetMesh"]


def _dev_tensor(a, dtype, device) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype).contiguous()


class DeviceTetMesh:
    """Connectivity of a tet mesh computed on the GPU; attributes are device tensors with the
    names and layouts of ``Mesh3D`` (``edges`` (2, N_e), ``tris`` (3, N_f), ``tet_to_edge`` (6, N_t),
    ``tet_to_tri`` (4, N_t), ``tri_to_edge`` (3, N_f), ``tri_to_tet`` (2, N_f, padded with -1234 as ``Mesh3D``),
    ``edge_lengths`` (N_e,))."""

    def __init__(self, nodes, tets, device=None):
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = dev
        self.nodes = _dev_tensor(nodes, torch.float64, dev)
        self.tets = _dev_tensor(tets, torch.int64, dev)
        if self.nodes.dim() != 2 or self.nodes.shape[0] != 3 or self.tets.dim() != 2 or self.tets.shape[0] != 4:
            raise ValueError("nodes must be (3, N_n) and tets (4, N_t)")
        nn, nt = self.nodes.shape[1], self.tets.shape[1]
        h = Handle.get(dev)
        c = ctypes.c_void_p()
        check(lib().emfem_mesh_connect_create(h.h, nn, nt, ptr(self.tets), ctypes.byref(c)),
              "emfem_mesh_connect_create")
        try:
            ne, nf = ctypes.c_int64(), ctypes.c_int64()
            check(lib().emfem_mesh_connect_info(c, ctypes.byref(ne), ctypes.byref(nf)), "emfem_mesh_connect_info")
            ne, nf = ne.value, nf.value
            i64 = dict(dtype=torch.int64, device=dev)
            self.edges = torch.empty((2, ne), **i64)
            self.tris = torch.empty((3, nf), **i64)
            self.tet_to_edge = torch.empty((6, nt), **i64)
            self.tet_to_tri = torch.empty((4, nt), **i64)
            self.tri_to_edge = torch.empty((3, nf), **i64)
            self.tri_to_tet = torch.empty((2, nf), **i64)
            self.edge_lengths = torch.empty(ne, dtype=torch.float64, device=dev)
            check(lib().emfem_mesh_connect_export(c, ptr(self.nodes), ptr(self.tets), ptr(self.edges),
                                                  ptr(self.tris), ptr(self.tet_to_edge), ptr(self.tet_to_tri),
                                                  ptr(self.tri_to_edge), ptr(self.tri_to_tet),
                                                  ptr(self.edge_lengths)), "emfem_mesh_connect_export")
            h.raise_on_device_status("emfem_mesh_connect_export")
        finally:
            lib().emfem_mesh_connect_destroy(c)

    @property
    def n_nodes(self) -> int:
        return self.nodes.shape[1]

    @property
    def n_tets(self) -> int:
        return self.tets.shape[1]

    @property
    def n_edges(self) -> int:
        return self.edges.shape[1]

    @property
    def n_tris(self) -> int:
        return self.tris.shape[1]

    def to_host(self) -> dict:
        """All connectivity arrays as host numpy arrays (keys = attribute names)."""
        keys = ("nodes", "tets", "edges", "tris", "tet_to_edge", "tet_to_tri", "tri_to_edge", "tri_to_tet",
                "edge_lengths")
        return {k: getattr(self, k).cpu().numpy() for k in keys}
