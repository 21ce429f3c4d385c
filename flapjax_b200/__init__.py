"""flapjax_b200: the FLAPJAX UVLM hot path on NVIDIA B200 (sm_100a).

The computation lives in ``libfj_uvlm.so`` (CUDA, C ABI declared in
``include/fj_uvlm.h``); this package is the host side with the reference's call surface.
"""
from .data_structures import AeroCase, ArrayList, GridDiscretisation
from .flowfields import Constant, FlowField, OneMinusCosine
from .kernels import biot_savart, biot_savart_cutoff, biot_savart_epsilon, cutoff_kernel
from .linear import (AeroInputUnflattened, AeroLinearResult, AeroOutputUnflattened, AeroStateUnflattened,
                     LinearInputProjection, LinearOutputProjection, LinearSystem, LinearUVLM)
from .polars import TabulatedPolar, tabulate
from .uvlm import UVLM, make_rectangular_grid

__all__ = [
    "AeroCase", "ArrayList", "GridDiscretisation", "Constant", "FlowField", "OneMinusCosine", "biot_savart",
    "biot_savart_cutoff", "biot_savart_epsilon", "cutoff_kernel", "UVLM", "make_rectangular_grid", "TabulatedPolar",
    "tabulate", "LinearUVLM", "LinearSystem", "LinearInputProjection", "LinearOutputProjection",
    "AeroInputUnflattened", "AeroStateUnflattened", "AeroOutputUnflattened", "AeroLinearResult",
]
