"""fiberlab_gpu -- B200-native GMMNLSE stepper (forward propagation and adjoint
gradient of FiberLab's interaction-picture solver) behind a C-ABI.

`problem` builds the tables on the host (FP64 numpy, mirroring the reference's
setup code); `solve` exposes the reference-shaped entry points; `_capi` binds
the CUDA library.  Importing this package does not load the CUDA library;
the first solve does, and fails loudly if it is missing.
"""
from . import problem
from .problem import ArgumentError, FiberProblem

__all__ = ["problem", "ArgumentError", "FiberProblem"]
__version__ = "0.1.0"
