"""B200-native NFGS (Gaussian-separated NFPT) reconstruction.

``NFGSSolverGPU`` keeps the reference solver's Python API; the numerical
work runs in the in-tree CUDA library ``libnfgs_b200.so`` (sm_100a).
"""

from .solver import NFGSSolverGPU

__all__ = ["NFGSSolverGPU", "release_cached_memory"]


def release_cached_memory(device: int = 0) -> None:
    """Hand back the device memory the library keeps reserved between
    solvers (and its idle pinned staging chunks) -- the counterpart of
    torch.cuda.empty_cache() for this library's allocations."""
    from . import _lib as L

    L.check(L.lib().nfgs_release_cached_memory(int(device)))
__version__ = "0.1.0"
