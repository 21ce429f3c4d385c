"""Biot-Savart kernel selectors (mirror ``flapjax.aero.utils.biot_savart*``,
aero/utils.py:580-648).

In the reference a kernel is a per-pair JAX function that ``UVLM(kernel=...)`` vmaps.
Here the pair loop lives in CUDA, so a kernel is a selector that names which formula
the library evaluates.  Each selector is still callable on one pair (or a batch of
pairs) and evaluates it on the GPU through ``fj_biot_savart``.
"""
from __future__ import annotations

import numpy as np

from . import _lib

EPSILON = 1e-7   # utils/constants.py:16
R_CUTOFF = 1e-4  # utils/constants.py:19


class KernelSpec:
    def __init__(self, kernel_id: int, name: str, r_cut: float = R_CUTOFF):
        self.kernel_id = kernel_id
        self.name = name
        self.r_cut = float(r_cut)

    def __repr__(self):
        extra = f", r_cut={self.r_cut:g}" if self.kernel_id == _lib.FJ_KERNEL_CUTOFF else ""
        return f"KernelSpec({self.name}{extra})"

    def __call__(self, x, y):
        """Kernel value for target(s) ``x`` (..., 3) and filament(s) ``y`` (..., 2, 3)."""
        import torch

        from .runtime import device_of

        x = np.asarray(x, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
        batch = np.broadcast_shapes(x.shape[:-1], y.shape[:-2])
        xb = np.array(np.broadcast_to(x, batch + (3,))).reshape(-1, 3)  # writable copies
        yb = np.array(np.broadcast_to(y, batch + (2, 3))).reshape(-1, 2, 3)
        dev = device_of(None)
        tx = torch.from_numpy(xb).to(dev)
        ty = torch.from_numpy(yb).to(dev)
        out = torch.empty_like(tx)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.call("fj_biot_savart", tx.data_ptr(), ty.data_ptr(), xb.shape[0], self.kernel_id, self.r_cut,
                  out.data_ptr(), stream)
        return out.cpu().numpy().reshape(batch + (3,))


biot_savart = KernelSpec(_lib.FJ_KERNEL_PLAIN, "biot_savart")
biot_savart_epsilon = KernelSpec(_lib.FJ_KERNEL_EPSILON, "biot_savart_epsilon")
biot_savart_cutoff = KernelSpec(_lib.FJ_KERNEL_CUTOFF, "biot_savart_cutoff")


def cutoff_kernel(radius: float) -> KernelSpec:
    """``biot_savart_cutoff`` with a vortex-core radius other than ``R_CUTOFF``."""
    return KernelSpec(_lib.FJ_KERNEL_CUTOFF, "biot_savart_cutoff", radius)


def resolve(kernel) -> KernelSpec:
    """Map ``UVLM(kernel=...)`` to a selector.  Accepts a KernelSpec, None (the default,
    epsilon kernel, aero/uvlm.py:280-285), or any callable whose ``__name__`` is one of
    the reference's kernel names (so the reference's function objects can be passed)."""
    if kernel is None:
        return biot_savart_epsilon
    if isinstance(kernel, KernelSpec):
        return kernel
    name = getattr(kernel, "__name__", None)
    table = {"biot_savart": biot_savart, "biot_savart_epsilon": biot_savart_epsilon,
             "biot_savart_cutoff": biot_savart_cutoff}
    if name in table:
        return table[name]
    raise TypeError(f"kernel {kernel!r} has no CUDA implementation; use a flapjax_b200.kernels selector")
