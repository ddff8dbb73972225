from .sparse_diffdmc import SparseDiffDMC, SparseDiffDMCOutput, SparseDMC

__all__ = ["SparseDiffDMC", "SparseDMC", "SparseDiffDMCOutput"]
