"""B200-native IISPH step of TurboSPHarticles behind its solver-backend interface.

`SimBackendB200` (backend.py) mirrors `Sim::I_SimBackend`
(source/simulation/core/backend_sim.h:194-261) over the C ABI of include/tsp_b200.h; the
compute runs in the in-tree CUDA library `_build/libtsp_b200.so` (sm_100a), which is
required: there is no CPU fallback.
"""
from .params import SimParams, dam_params  # noqa: F401
from .state import UniversalSimState  # noqa: F401
from . import abi, scene  # noqa: F401

__all__ = ["SimParams", "dam_params", "UniversalSimState", "abi", "scene"]


def __getattr__(name):
    if name == "SimBackendB200":
        from .backend import SimBackendB200
        return SimBackendB200
    raise AttributeError(name)
