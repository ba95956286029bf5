"""B200-native NFGS (Gaussian-separated NFPT) reconstruction.

``NFGSSolverGPU`` keeps the reference solver's Python API; the numerical
work runs in the in-tree CUDA library ``libnfgs_b200.so`` (sm_100a).
"""

from .solver import NFGSSolverGPU

__all__ = ["NFGSSolverGPU"]
__version__ = "0.1.0"
