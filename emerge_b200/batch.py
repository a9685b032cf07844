"""Many uneven meshes assembled in one launch.

The reference assembles one mesh per ``tet_mass_stiffness_matrices`` call (``ASM/curlcurl.py:145-173``).
:class:`MeshBatch` concatenates a list of meshes into one disjoint union: node ids of mesh k are
offset by the node counts of meshes 0..k-1.  It computes the union's connectivity on the device
(:class:`connectivity.DeviceTetMesh`), builds one symbolic plan and assembles E and B of every mesh
with one launch of the fused kernel.

Union ids keep each mesh contiguous.  Unique edges and triangles are sorted lexicographically by node
id, and the offsets increase with k, so mesh k's edges form one contiguous range of the union's edges
and its triangles one range of the union's triangles.  Its DOFs are therefore the four ranges
[edges_k | faces_k | edges_k + H | faces_k + H] (``elements/nedelec2.py:42-58``).  Each row of the
union CSR lists exactly mesh k's columns, in mesh k's own order.  Each value is summed over the same
tets in the same order as a separate assembly.  :meth:`MeshBatch.csr` therefore returns every mesh's
matrices bit for bit equal to assembling that mesh alone.

``ASM/`` = ``src/emerge/_emerge/physics/microwave/assembly/``.
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.sparse import csr_matrix

from .assembly import CsrPlan, DeviceMesh
from .connectivity import DeviceTetMesh

__all__ = ["MeshBatch"]


class MeshBatch:
    def __init__(self, meshes, device=None):
        """meshes: list of (nodes (3, N_n), tets (4, N_t)) in Mesh3D layouts (host or device)."""
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = dev
        nodes, tets, self.node_off, self.tet_off = [], [], [0], [0]
        for nd, tt in meshes:
            nd = torch.as_tensor(np.asarray(nd) if not isinstance(nd, torch.Tensor) else nd).to(dev, torch.float64)
            tt = torch.as_tensor(np.asarray(tt) if not isinstance(tt, torch.Tensor) else tt).to(dev, torch.int64)
            nodes.append(nd)
            tets.append(tt + self.node_off[-1])
            self.node_off.append(self.node_off[-1] + nd.shape[1])
            self.tet_off.append(self.tet_off[-1] + tt.shape[1])
        self.n_meshes = len(meshes)
        self.mesh = DeviceTetMesh(torch.cat(nodes, dim=1), torch.cat(tets, dim=1), dev)
        self.dmesh = DeviceMesh(self.mesh, None, dev)
        self.plan = CsrPlan(self.dmesh)
        # per-mesh entity ranges: edges/tris whose first (smallest) node lies in the mesh's node range
        no = torch.tensor(self.node_off, device=dev)
        self.edge_off = torch.searchsorted(self.mesh.edges[0].contiguous(), no).cpu().numpy()
        self.tri_off = torch.searchsorted(self.mesh.tris[0].contiguous(), no).cpu().numpy()
        self.E = self.B = None

    @property
    def n_tets(self) -> int:
        return self.tet_off[-1]

    def assemble(self, er: torch.Tensor, ur: torch.Tensor):
        """One fused launch for every mesh; er/ur (3, 3, total tets) complex (mesh order)."""
        self.E, self.B = self.plan.assemble(er, ur, self.E, self.B)
        return self.E, self.B

    def dof_ranges(self, k: int) -> list[tuple[int, int]]:
        """Mesh k's DOFs in the union numbering: [edges | faces | edges + H | faces + H]."""
        ne, nf = self.dmesh.n_edges, self.dmesh.n_tris
        H = ne + nf
        e0, e1 = int(self.edge_off[k]), int(self.edge_off[k + 1])
        t0, t1 = int(self.tri_off[k]), int(self.tri_off[k + 1])
        return [(e0, e1), (ne + t0, ne + t1), (H + e0, H + e1), (H + ne + t0, H + ne + t1)]

    def csr(self, k: int, which: str = "E") -> csr_matrix:
        """Mesh k's E or B as a SciPy CSR in its own DOF numbering (host copy)."""
        vals = (self.E if which == "E" else self.B).cpu().numpy()
        indptr, indices = self.plan.host_pattern()
        ranges = self.dof_ranges(k)
        rows = np.concatenate([np.arange(a, b) for a, b in ranges])
        n = len(rows)
        local = np.full(self.plan.n_field, -1, dtype=np.int64)
        local[rows] = np.arange(n)
        starts, ends = indptr[rows], indptr[rows + 1]
        sel = np.concatenate([np.arange(s, e) for s, e in zip(starts, ends)])
        cols = local[indices[sel]]
        if (cols < 0).any():
            raise RuntimeError("MeshBatch: a row couples two meshes (inputs are not disjoint)")
        new_ptr = np.concatenate([[0], np.cumsum(ends - starts)])
        return csr_matrix((vals[sel], cols.astype(np.int32), new_ptr.astype(np.int32)), shape=(n, n))
