"""B200-native multi-way joins: the AMHJ multi-way hash join and the ALFTJ
leapfrog triejoin of RapidsAtHKUST/AccMultiwayJoins, as hand-written sm_100a
CUDA behind a C ABI (include/amj.h, libamj.so), with this package as the
Python host layer."""
from ._lib import AmjError, load as load_library  # noqa: F401
from .core import Batch, BatchRun, Context, Relation, Result, Server, ServeResult, cuda_device_available  # noqa: F401
from . import data  # noqa: F401

__all__ = ["AmjError", "Batch", "BatchRun", "Context", "Server", "ServeResult", "Relation", "Result", "cuda_device_available", "data", "load_library"]
