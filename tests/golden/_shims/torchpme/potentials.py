"""Potential base class: kernel_from_k_sq forwards to lr_from_k_sq."""
import torch


class Potential(torch.nn.Module):
    def __init__(self, smearing=None, exclusion_radius=None):
        super().__init__()
        self.smearing = smearing
        self.exclusion_radius = exclusion_radius

    def kernel_from_k_sq(self, k_sq):
        return self.lr_from_k_sq(k_sq)
