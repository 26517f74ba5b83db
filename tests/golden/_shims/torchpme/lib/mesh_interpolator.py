"""MeshInterpolator base: attributes read by MeshInterpolatorD3.points_to_mesh."""
import torch

from oracle.torchpme_shim import mesh_weights


class MeshInterpolator:
    def __init__(self, cell, ns_mesh, interpolation_nodes, method):
        self.interpolation_nodes = int(interpolation_nodes)
        self.method = method
        self.cell = cell
        self.ns_mesh = ns_mesh
        self._dtype = cell.dtype
        self._device = cell.device
        self.update(cell, ns_mesh)

    def update(self, cell=None, ns_mesh=None):
        if cell is not None:
            self.cell = cell
            self.inverse_cell = torch.linalg.inv(cell)
        if ns_mesh is not None:
            self.ns_mesh = ns_mesh

    def compute_weights(self, positions):
        p = self.interpolation_nodes
        w, base = mesh_weights(positions, self.inverse_cell, self.ns_mesh, p, self.method)
        self.interpolation_weights = w                                   # (p, N, 3)
        ar = torch.arange(p, device=positions.device)
        sx, sy, sz = torch.meshgrid(ar, ar, ar, indexing="ij")
        self.x_shifts, self.y_shifts, self.z_shifts = sx.flatten(), sy.flatten(), sz.flatten()
        nodes = base.unsqueeze(0) + ar.view(p, 1, 1)                     # (p, N, 3)
        self.x_indices = nodes[self.x_shifts, :, 0] % int(self.ns_mesh[0])
        self.y_indices = nodes[self.y_shifts, :, 1] % int(self.ns_mesh[1])
        self.z_indices = nodes[self.z_shifts, :, 2] % int(self.ns_mesh[2])
