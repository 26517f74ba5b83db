"""fourierd3_b200 -- B200-native FourierD3 dispersion (DFT-D3(BJ) in reciprocal space).

Public surface (drop-in for the reference package ``fourierd3``):
    FourierD3               torch module, forward(positions, edge_index, shifts) -> energy
    FourierD3ASECalculator  ASE calculator (energy, forces, stress)
    forward                 functional (positions, cell, numbers) -> (energy, forces, stress)
    neighbour_list          device cell-list neighbour build, (i, j, S) like matscipy "ijS"
All compute runs in libfd3.so (hand-written sm_100a CUDA kernels + cuFFT).
"""
from fourierd3_b200.calculator import FourierD3ASECalculator
from fourierd3_b200.core import FourierD3
from fourierd3_b200.engine import neighbour_list
from fourierd3_b200.batch import D3Batch
from fourierd3_b200.functional import D3Model, forward, forward_batch

__all__ = ("FourierD3", "FourierD3ASECalculator", "forward", "forward_batch", "neighbour_list", "D3Model",
           "D3Batch")
