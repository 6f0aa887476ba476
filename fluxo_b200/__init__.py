"""B200-native (sm_100a, FP64) DGSEM right-hand side and LSERK time step of FLUXO.

The compute path is ``libfluxo_gpu.so`` (hand-written CUDA, C ABI in ``include/fluxo_gpu.h``);
this package is the Python host side that mirrors the reference's operator interface.
"""
from ._lib import FluxoError, load  # noqa: F401
from .solver import DGOperator, Fluxo, box_mesh, exact_func, make_cfg  # noqa: F401
