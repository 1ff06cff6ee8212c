"""erf_b200: B200-native multirate RK3 dycore (ERF hot path) behind a C-ABI.

    from erf_b200 import cases, config, Dycore
"""
from . import config, cases
from .dycore import Dycore, load_library, LIB_PATH, EXPORTS, KERNEL_SLOTS

__all__ = ["config", "cases", "Dycore", "load_library", "LIB_PATH", "EXPORTS"]
