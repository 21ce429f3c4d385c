"""JAX binding of the C ABI: ``jax.ffi`` custom calls with ``jax.custom_vjp`` rules.

It covers the two operations of the reference's aero step that this library replaces at
function level:

* ``compute_v_ind`` (aero/aic.py:248-310, looked up by name at aero/uvlm.py:15):
  ``fj_vind`` per source lattice, with the VJP from ``fj_vind_vjp``;
* the dense solve ``jnp.linalg.solve(aic, b)`` (aero/uvlm.py:985): ``fj_lu_factor`` +
  ``fj_lu_solve``, whose VJP reuses the factors in ``fj_lu_solve_t``
  (db = A^-T g, dA = -db x^T).

The module imports without JAX (``available()`` is then False and every other function
raises); it needs JAX with x64 enabled and the handler library ``libfj_xla.so`` built from
``flapjax_b200/xla/fj_xla.cc`` (``python -m flapjax_b200.build --xla``, which reads
jaxlib's FFI headers).  ``install()`` rebinds ``flapjax.aero.uvlm.compute_v_ind`` so the
reference's own UVLM calls the CUDA sums.  The VJP is the FP64 epsilon-kernel adjoint
(``fj_vind_vjp``); mirror images are supported in the forward only.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from . import _lib
from .kernels import resolve

try:  # optional: the module is importable (and reviewable) where JAX is absent
    import jax
    import jax.numpy as jnp
except ImportError:  # pragma: no cover - exercised on machines without JAX
    jax = None
    jnp = None

XLA_LIB = Path(__file__).resolve().parent / "_lib" / "libfj_xla.so"
_TARGETS = {"fj_vind": "FjVInd", "fj_vind_vjp": "FjVIndVjp", "fj_lu_factor": "FjLuFactor",
            "fj_lu_solve": "FjLuSolve"}
_registered = False


def available() -> bool:
    """True where JAX imports and the handler library has been built."""
    return jax is not None and XLA_LIB.exists()


def _require():
    if jax is None:
        raise RuntimeError("flapjax_b200.fj_jax needs JAX (jax.ffi), which is not installed")
    if not XLA_LIB.exists():
        raise RuntimeError(f"{XLA_LIB} is missing: build it with `python -m flapjax_b200.build --xla`")


def register(lib_path: str | Path | None = None) -> None:
    """Register the four FFI targets for the CUDA platform (idempotent)."""
    global _registered
    _require()
    if _registered:
        return
    lib = C.CDLL(str(lib_path or XLA_LIB))
    for name, sym in _TARGETS.items():
        jax.ffi.register_ffi_target(name, jax.ffi.pycapsule(getattr(lib, sym)), platform="CUDA")
    _registered = True


def _ws_vind(n_targets, rows, cols, mirror, precision):
    n = C.c_size_t()
    _lib.call("fj_vind_workspace_size", int(n_targets), (C.c_int * 1)(rows), (C.c_int * 1)(cols), 1, int(mirror),
              int(precision), C.byref(n))
    return max(1, int(n.value))


def _ws_vjp(n_targets, rows, cols):
    n = C.c_size_t()
    _lib.call("fj_vind_vjp_workspace_size", int(n_targets), (C.c_int * 1)(rows), (C.c_int * 1)(cols), 1, 0,
              C.byref(n))
    return max(1, int(n.value))


def _ws_lu(n):
    b = C.c_size_t()
    _lib.call("fj_lu_workspace_size", int(n), C.byref(b))
    return max(1, int(b.value))


def _vind_one(c, zeta, gamma, kernel_id, r_cut, precision, mirror):
    """Velocity of one lattice at the flat targets c (n, 3)."""
    rows, cols = gamma.shape
    ws = jnp.zeros((_ws_vind(c.shape[0], rows, cols, mirror is not None, precision),), jnp.uint8)
    m = jnp.zeros(6) if mirror is None else jnp.concatenate([jnp.ravel(mirror[0]), jnp.ravel(mirror[1])])
    return jax.ffi.ffi_call("fj_vind", jax.ShapeDtypeStruct(c.shape, jnp.float64))(
        c, zeta, gamma, ws, mirror=tuple(float(x) for x in m), has_mirror=int(mirror is not None),
        kernel=int(kernel_id), r_cut=float(r_cut), precision=int(precision))


def _vind_vjp_one(c, zeta, gamma, lam, kernel_id, r_cut):
    rows, cols = gamma.shape
    ws = jnp.zeros((_ws_vjp(c.shape[0], rows, cols),), jnp.uint8)
    out = (jax.ShapeDtypeStruct(c.shape, jnp.float64), jax.ShapeDtypeStruct(zeta.shape, jnp.float64),
           jax.ShapeDtypeStruct(gamma.shape, jnp.float64))
    return jax.ffi.ffi_call("fj_vind_vjp", out)(c, zeta, gamma, lam, ws, kernel=int(kernel_id), r_cut=float(r_cut))


def make_vind(kernel_id: int, r_cut: float, precision: int = 0):
    """v(c, zeta, gamma) for one lattice, differentiable through fj_vind_vjp."""
    _require()

    @jax.custom_vjp
    def vind(c, zeta, gamma):
        return _vind_one(c, zeta, gamma, kernel_id, r_cut, precision, None)

    def fwd(c, zeta, gamma):
        return vind(c, zeta, gamma), (c, zeta, gamma)

    def bwd(res, lam):
        return _vind_vjp_one(*res, lam, kernel_id, r_cut)

    vind.defvjp(fwd, bwd)
    return vind


def compute_v_ind(cs, zetas, gammas, kernels, mirror_point, mirror_normal, batch_size=None, precision=0):
    """Drop-in for the reference's ``compute_v_ind`` (aero/aic.py:248-310): same arguments
    (``batch_size`` is ignored), same Array / ArrayList return."""
    register()
    single = not isinstance(cs, (list, tuple))
    out = []
    mirror = None if mirror_point is None or mirror_normal is None else (mirror_point, mirror_normal)
    for c in ([cs] if single else cs):
        flat = jnp.reshape(c, (-1, 3))
        v = jnp.zeros_like(flat)
        for zeta, gamma, kernel in zip(zetas, gammas, kernels):
            if gamma.size == 0:
                continue
            spec = resolve(kernel)
            if mirror is None:
                v = v + make_vind(spec.kernel_id, spec.r_cut, precision)(flat, zeta, gamma)
            else:
                v = v + _vind_one(flat, zeta, gamma, spec.kernel_id, spec.r_cut, precision, mirror)
        out.append(jnp.reshape(v, c.shape))
    if single:
        return out[0]
    return type(cs)(out)


def solve(a, b):
    """``jnp.linalg.solve(a, b)`` for one right-hand side on the getrf factors."""
    register()
    return _solve_fwd(a, b)[0]


def _solve_fwd(a, b):
    n = a.shape[0]
    lu, piv = jax.ffi.ffi_call("fj_lu_factor", (jax.ShapeDtypeStruct(a.shape, jnp.float64),
                                                jax.ShapeDtypeStruct((n,), jnp.int32)))(
        a, jnp.zeros((_ws_lu(n),), jnp.uint8))
    x = _lu_solve(lu, piv, b, 0)
    return x, (lu, piv, x)


def _lu_solve(lu, piv, b, transpose):
    n = lu.shape[0]
    return jax.ffi.ffi_call("fj_lu_solve", jax.ShapeDtypeStruct(b.shape, jnp.float64))(
        lu, piv, b, jnp.zeros((_ws_lu(n),), jnp.uint8), transpose=int(transpose))


def _solve_bwd(res, g):
    lu, piv, x = res
    bbar = _lu_solve(lu, piv, g, 1)
    return -jnp.outer(bbar, x), bbar


if jax is not None:
    solve = jax.custom_vjp(solve)
    solve.defvjp(_solve_fwd, _solve_bwd)


def install(uvlm_module=None) -> None:
    """Rebind ``compute_v_ind`` in the reference's ``flapjax.aero.uvlm`` (the name the
    UVLM class calls at aero/uvlm.py:920, 969, 1025, 1622, 1726, 1891)."""
    register()
    if uvlm_module is None:
        import importlib

        uvlm_module = importlib.import_module("flapjax.aero.uvlm")
    uvlm_module.compute_v_ind = compute_v_ind
