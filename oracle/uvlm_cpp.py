"""The FP64 oracle with its pair-heavy sums in C++/OpenMP (TEST INFRASTRUCTURE AND CPU
BASELINE ONLY).

``UVLMCpp`` is ``uvlm_ref.UVLMRef`` with ``compute_v_ind`` and ``compute_aic_solve``
(aero/aic.py:11-310) evaluated by ``uvlm_ref_cpu.cpp`` (OpenMP over target points, SIMD
over filaments); the O(M N) arithmetic stays in NumPy and the dense solve in LAPACK, as
the reference's XLA CPU path calls LAPACK for jnp.linalg.solve (aero/uvlm.py:985).
Build: ``make -C oracle``.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import uvlm_ref as R

_LIB = Path(__file__).resolve().parent / "_lib" / "libuvlm_ref_cpu.so"
_KERNEL = {R.KERNEL_EPSILON: 0, R.KERNEL_CUTOFF: 1, R.KERNEL_PLAIN: 2}
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not _LIB.exists():
            raise RuntimeError(f"{_LIB} not built (make -C oracle)")
        _lib = C.CDLL(str(_LIB))
        P, I64, I, D = C.c_void_p, C.c_int64, C.c_int, C.c_double
        _lib.uvref_vind.argtypes = [P, I64, P, P, P, P, I, P, P, I, D, P]
        _lib.uvref_aic.argtypes = [P, P, I64, P, P, P, I, P, P, P, P, I, D, P]
        _lib.uvref_set_threads.argtypes = [I]
    return _lib


def max_threads() -> int:
    return lib().uvref_max_threads()


def set_threads(n: int) -> None:
    lib().uvref_set_threads(int(n))


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptrs(arrs):
    return (C.c_void_p * max(1, len(arrs)))(*[a.ctypes.data for a in arrs])


def _ints(v):
    return (C.c_int * max(1, len(v)))(*v)


def _mirror(mirror):
    if mirror is None:
        return None, None, ()
    p, n = _c(mirror[0]), _c(mirror[1])
    return p.ctypes.data, n.ctypes.data, (p, n)


def compute_v_ind(cs, zetas, gammas, kernel, mirror=None, r_cut=R.R_CUTOFF):
    t = _c(cs).reshape(-1, 3)
    zs = [_c(z) for z in zetas]
    gs = [_c(g) for g in gammas]
    out = np.empty_like(t)
    mp, mn, keep = _mirror(mirror)
    rc = lib().uvref_vind(t.ctypes.data, t.shape[0], _ptrs(zs), _ptrs(gs), _ints([g.shape[0] for g in gs]),
                          _ints([g.shape[1] for g in gs]), len(zs), mp, mn, _KERNEL[kernel], float(r_cut),
                          out.ctypes.data)
    if rc:
        raise RuntimeError("uvref_vind failed")
    return out.reshape(np.shape(cs))


def compute_aic_solve(cs, ns, zetas_b, zetas_w, kernel, mirror=None, r_cut=R.R_CUTOFF):
    c = np.concatenate([_c(x).reshape(-1, 3) for x in cs])
    n = np.concatenate([_c(x).reshape(-1, 3) for x in ns])
    zb = [_c(z) for z in zetas_b]
    m = [z.shape[0] - 1 for z in zb]
    nn = [z.shape[1] - 1 for z in zb]
    zw = None if zetas_w is None else [_c(z) for z in zetas_w]
    out = np.empty((c.shape[0], sum(a * b for a, b in zip(m, nn))))
    mp, mn, keep = _mirror(mirror)
    rc = lib().uvref_aic(c.ctypes.data, n.ctypes.data, c.shape[0], _ptrs(zb), _ints(m), _ints(nn), len(zb),
                         None if zw is None else _ptrs(zw), None if zw is None else _ints([z.shape[0] - 1 for z in zw]),
                         mp, mn, _KERNEL[kernel], float(r_cut), out.ctypes.data)
    if rc:
        raise RuntimeError("uvref_aic failed")
    return out


class UVLMCpp(R.UVLMRef):
    """``UVLMRef`` with the induced-velocity sums and the AIC assembly in C++/OpenMP."""

    def v_ind(self, x, zetas, gammas):
        return compute_v_ind(x, zetas, gammas, self.kernel, self.mirror, self.r_cut)

    def aic_solve(self, cs, ns, zetas_b, zetas_w):
        return compute_aic_solve(cs, ns, zetas_b, zetas_w, self.kernel, self.mirror, self.r_cut)
