"""B200-native FLIP liquid step of 水理ラボ (suiri-lab) behind the C-ABI library ``libsuiri_cuda.so``.

``Tank`` is one scene on the GPU (the plain drop-in path), ``Batch`` steps many tanks with shared launches.
"""
from . import native, workloads  # noqa: F401
from .tank import Batch, Tank  # noqa: F401
from .serve import Server  # noqa: F401
