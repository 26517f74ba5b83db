"""KSpaceFilter base: update() -> _prep_kvectors() then the kernel on |k|."""
import torch


class KSpaceFilter(torch.nn.Module):
    def __init__(self, cell, ns_mesh, kernel, fft_norm="ortho", ifft_norm="ortho"):
        super().__init__()
        self._fft_norm = fft_norm
        self._ifft_norm = ifft_norm
        self.kernel = kernel
        self.cell = cell
        self.ns_mesh = ns_mesh
        self.update(cell, ns_mesh)

    def update(self, cell=None, ns_mesh=None):
        self._prep_kvectors(cell, ns_mesh)
        self._kfilter = self.kernel.kernel_from_k_sq(self._k_sq)
