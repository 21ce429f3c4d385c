"""torch.autograd bindings of the hand-written adjoint kernels, used for gradient checks.

``induced_velocity``: v = compute_v_ind(targets; lattice, gamma) (aero/aic.py:208-310)
through ``fj_vind``, with ``fj_vind_vjp`` as its backward (vertex, circulation and target
cotangents in one pass).  ``dense_solve``: x = solve(A, b) (aero/uvlm.py:985) through
``fj_lu_factor`` / ``fj_lu_solve``; its backward reuses the kept getrf factors in the
transpose solve ``fj_lu_solve_t``: b_bar = A^-T x_bar, A_bar = -b_bar x^T.

Both run in FP64 on the CUDA device of their inputs and exist so that
``torch.autograd.gradcheck`` can compare the hand-written adjoints with central
differences; the reference differentiates the same functions with ``jax.vjp``.  There is
no CPU path: the library raises when its CUDA extension is missing.
"""
from __future__ import annotations

import ctypes as C

from . import _lib


def _stream(t):
    import torch

    return torch.cuda.current_stream(t.device).cuda_stream


def _workspace(nbytes, device):
    import torch

    return torch.empty(max(1, int(nbytes)), dtype=torch.uint8, device=device)


def _function_classes():
    import torch

    class InducedVelocity(torch.autograd.Function):
        @staticmethod
        def forward(ctx, targets, zeta, gamma, kernel, r_cut):
            targets, zeta, gamma = targets.contiguous(), zeta.contiguous(), gamma.contiguous()
            rows, cols = (C.c_int * 1)(gamma.shape[0]), (C.c_int * 1)(gamma.shape[1])
            zp, gp = (C.c_void_p * 1)(zeta.data_ptr()), (C.c_void_p * 1)(gamma.data_ptr())
            nt = targets.numel() // 3
            nb = C.c_size_t()
            _lib.call("fj_vind_workspace_size", nt, rows, cols, 1, 0, _lib.FJ_PREC_FP64, C.byref(nb))
            ws = _workspace(nb.value, targets.device)
            v = torch.empty_like(targets)
            _lib.call("fj_vind", targets.data_ptr(), nt, zp, gp, rows, cols, 1, None, None, kernel, r_cut,
                      _lib.FJ_PREC_FP64, v.data_ptr(), ws.data_ptr(), ws.numel(), _stream(targets))
            ctx.save_for_backward(targets, zeta, gamma)
            ctx.kernel, ctx.r_cut = kernel, r_cut
            return v

        @staticmethod
        def backward(ctx, v_bar):
            targets, zeta, gamma = ctx.saved_tensors
            rows, cols = (C.c_int * 1)(gamma.shape[0]), (C.c_int * 1)(gamma.shape[1])
            zp, gp = (C.c_void_p * 1)(zeta.data_ptr()), (C.c_void_p * 1)(gamma.data_ptr())
            nt = targets.numel() // 3
            lam = v_bar.contiguous()
            t_bar, z_bar, g_bar = torch.zeros_like(targets), torch.zeros_like(zeta), torch.zeros_like(gamma)
            zbp, gbp = (C.c_void_p * 1)(z_bar.data_ptr()), (C.c_void_p * 1)(g_bar.data_ptr())
            nb = C.c_size_t()
            _lib.call("fj_vind_vjp_workspace_size", nt, rows, cols, 1, 0, C.byref(nb))
            ws = _workspace(nb.value, targets.device)
            _lib.call("fj_vind_vjp", targets.data_ptr(), nt, zp, gp, rows, cols, 1, None, None, ctx.kernel,
                      ctx.r_cut, lam.data_ptr(), t_bar.data_ptr(), zbp, gbp, ws.data_ptr(), ws.numel(),
                      _stream(targets))
            return t_bar, z_bar, g_bar, None, None

    class DenseSolve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, a, b):
            n = b.numel()
            lu = a.contiguous().clone()
            piv = torch.empty(n, dtype=torch.int32, device=a.device)
            nb = C.c_size_t()
            _lib.call("fj_lu_workspace_size", n, C.byref(nb))
            ws = _workspace(nb.value, a.device)
            _lib.call("fj_lu_factor", lu.data_ptr(), n, piv.data_ptr(), ws.data_ptr(), ws.numel(), _stream(a))
            x = b.contiguous().clone()
            _lib.call("fj_lu_solve", lu.data_ptr(), n, piv.data_ptr(), x.data_ptr(), ws.data_ptr(), ws.numel(),
                      _stream(a))
            ctx.save_for_backward(lu, piv, x)
            return x

        @staticmethod
        def backward(ctx, x_bar):
            lu, piv, x = ctx.saved_tensors
            n = x.numel()
            nb = C.c_size_t()
            _lib.call("fj_lu_workspace_size", n, C.byref(nb))
            ws = _workspace(nb.value, x.device)
            b_bar = x_bar.contiguous().clone()
            _lib.call("fj_lu_solve_t", lu.data_ptr(), n, piv.data_ptr(), b_bar.data_ptr(), ws.data_ptr(),
                      ws.numel(), _stream(x))
            return -torch.outer(b_bar, x), b_bar

    return InducedVelocity, DenseSolve


_CLASSES = None


def _classes():
    global _CLASSES
    if _CLASSES is None:
        _CLASSES = _function_classes()
    return _CLASSES


def induced_velocity(targets, zeta, gamma, kernel=_lib.FJ_KERNEL_EPSILON, r_cut=0.0):
    """v (n, 3) induced at targets (n, 3) by one vortex lattice zeta (R+1, C+1, 3) with ring
    circulations gamma (R, C); FP64 CUDA tensors.  Differentiable in all three."""
    return _classes()[0].apply(targets, zeta, gamma, kernel, r_cut)


def dense_solve(a, b):
    """x with A x = b (A (n, n), b (n,), FP64 CUDA tensors), differentiable in A and b."""
    return _classes()[1].apply(a, b)
