"""B200-native FLIP liquid step of 水理ラボ (suiri-lab) behind the C-ABI library ``libsuiri_cuda.so``."""
from . import workloads  # noqa: F401
