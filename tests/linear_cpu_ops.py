"""CPU stand-ins for the device operations of ``flapjax_b200.linear`` (test-only).

The linear model's assembly (``flapjax_b200.linear._assemble``) calls a small set of
device operations: ring influence and vertex Jacobians of the Biot-Savart sum, induced
velocities and their target gradients, the AIC factorisation and solves.  These classes
give the same operations on the CPU from the FP64 oracle (velocities exactly, the
Jacobians by central differences of the oracle's sums), so that the chain rule and the
block bookkeeping of the assembly can be checked here against the reference's own
Jacobians, without a GPU.  The product never uses them: ``LinearUVLM`` builds its device
operations from the CUDA library and has no CPU path.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg
import torch

from flapjax_b200 import _lib
from oracle import uvlm_ref as R

_KER = {_lib.FJ_KERNEL_EPSILON: R.KERNEL_EPSILON, _lib.FJ_KERNEL_CUTOFF: R.KERNEL_CUTOFF}


class OracleOps:
    torch = torch

    def __init__(self, mirror=None, h=1e-6):
        self.mirror = None if mirror is None else (np.asarray(mirror[0], float),
                                                   np.asarray(mirror[1], float) / np.linalg.norm(mirror[1]))
        self.h = h

    def tensor(self, a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64))

    def zeros(self, *shape):
        return torch.zeros(shape, dtype=torch.float64)

    def _v(self, x, lats, kernel, r_cut):
        return R.compute_v_ind(x, [np.asarray(z) for z, _ in lats], [np.asarray(g) for _, g in lats], _KER[kernel],
                               self.mirror, r_cut)

    def ring(self, out, col0, targets, normals, zeta, kernel, r_cut):
        x = targets.numpy()
        z = zeta.numpy()
        rows, cols = z.shape[0] - 1, z.shape[1] - 1
        for r in range(rows * cols):
            g = np.zeros((rows, cols))
            g.flat[r] = 1.0
            v = self._v(x, [(z, g)], kernel, r_cut)
            if normals is None:
                out[:, col0 + r] = torch.as_tensor(v.reshape(-1))
            else:
                out[:, col0 + r] = torch.as_tensor(np.einsum("ij,ij->i", v, normals.numpy()))

    def vertex(self, out, col0, targets, normals, zeta, gamma, kernel, r_cut):
        x = targets.numpy()
        z = zeta.numpy().copy()
        g = gamma.numpy()
        for j in range(z.size):
            zp, zm = z.copy(), z.copy()
            zp.flat[j] += self.h
            zm.flat[j] -= self.h
            d = (self._v(x, [(zp, g)], kernel, r_cut) - self._v(x, [(zm, g)], kernel, r_cut)) / (2 * self.h)
            if normals is None:
                out[:, col0 + j] = torch.as_tensor(d.reshape(-1))
            else:
                out[:, col0 + j] = torch.as_tensor(np.einsum("ij,ij->i", d, normals.numpy()))

    def vind(self, targets, lats, kernel, r_cut):
        return torch.as_tensor(self._v(targets.numpy(), [(z.numpy(), g.numpy()) for z, g in lats], kernel, r_cut))

    def vind_grad_t(self, targets, lats, kernel, r_cut, lam):
        x = targets.numpy()
        L = [(z.numpy(), g.numpy()) for z, g in lats]
        lm = lam.numpy()
        out = np.zeros_like(x)
        for b in range(3):
            xp, xm = x.copy(), x.copy()
            xp[:, b] += self.h
            xm[:, b] -= self.h
            d = (self._v(xp, L, kernel, r_cut) - self._v(xm, L, kernel, r_cut)) / (2 * self.h)
            out[:, b] = np.einsum("ij,ij->i", lm, d)
        return torch.as_tensor(out)

    def aic_factor(self, zetas_b, kernel, r_cut):
        zs = [z.numpy() for z in zetas_b]
        cs = [R.compute_surf_c(z) for z in zs]
        ns = [R.compute_surf_nc(z) for z in zs]
        a = R.compute_aic_solve(cs, ns, zs, None, _KER[kernel], self.mirror, r_cut)
        return scipy.linalg.lu_factor(a), None

    def solve(self, lu, piv, b):
        return torch.as_tensor(scipy.linalg.lu_solve(lu, b.numpy()))

    def solve_many(self, lu, piv, b):
        b[...] = torch.as_tensor(scipy.linalg.lu_solve(lu, b.numpy()))
