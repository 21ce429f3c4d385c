"""fj_vind_noalloc: induced velocities for callers that cannot allocate device memory.

Such callers (a plugin host that owns the device memory pool, a real-time loop that may
not block in cudaMalloc) cannot provide fj_vind's workspace; fj_vind_noalloc uses a fixed
8 MiB array inside the library instead.  Checked against fj_vind (which takes a caller
workspace) and against the FP64 oracle on two consecutive calls with different inputs, in
FP64 (1e-10 normwise, the FP64 bar of the other tests) and in the mixed path (2e-6, the
FP32 velocity bar); with a mirror plane; with so many targets that fewer splits fit in the
array than fj_vind would use; and its refusal of sizes beyond the array.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import uvlm_ref as R

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(dev)


def _lattices(rng, shapes):
    out = []
    for r, c in shapes:
        z = np.zeros((r + 1, c + 1, 3))
        z[..., 0] = np.linspace(0, 1, r + 1)[:, None] + 0.01 * rng.normal(size=(r + 1, c + 1))
        z[..., 1] = np.linspace(0, 3, c + 1)[None, :] + 0.01 * rng.normal(size=(r + 1, c + 1))
        z[..., 2] = 0.05 * rng.normal(size=(r + 1, c + 1))
        out.append((z, rng.normal(size=(r, c))))
    return out


def _mirror_args(mirror):
    if mirror is None:
        return None, None
    return (C.c_double * 3)(*mirror[0]), (C.c_double * 3)(*mirror[1])


def _args(dev, targets, lats):
    zs = [_t(z, dev) for z, _ in lats]
    gs = [_t(g, dev) for _, g in lats]
    n = len(lats)
    return dict(
        keep=(zs, gs),
        tt=_t(targets, dev),
        zp=(C.c_void_p * n)(*[z.data_ptr() for z in zs]),
        gp=(C.c_void_p * n)(*[g.data_ptr() for g in gs]),
        rows=(C.c_int * n)(*[z.shape[0] - 1 for z, _ in lats]),
        cols=(C.c_int * n)(*[z.shape[1] - 1 for z, _ in lats]),
        n=n,
    )


def _with_workspace(dev, a, n_t, kernel, r_cut, precision, mirror=None):
    import torch

    from flapjax_b200 import _lib

    mp, mn = _mirror_args(mirror)
    nbytes = C.c_size_t()
    _lib.call("fj_vind_workspace_size", n_t, a["rows"], a["cols"], a["n"], int(mirror is not None), precision,
              C.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    out = torch.empty((n_t, 3), dtype=torch.float64, device=dev)
    _lib.call("fj_vind", a["tt"].data_ptr(), n_t, a["zp"], a["gp"], a["rows"], a["cols"], a["n"], mp, mn, kernel,
              r_cut, precision, out.data_ptr(), ws.data_ptr(), ws.numel(), torch.cuda.current_stream(dev).cuda_stream)
    return out.cpu().numpy()


def _no_alloc(dev, a, n_t, kernel, r_cut, precision, mirror=None):
    import torch

    from flapjax_b200 import _lib

    mp, mn = _mirror_args(mirror)
    out = torch.empty((n_t, 3), dtype=torch.float64, device=dev)
    _lib.call("fj_vind_noalloc", a["tt"].data_ptr(), n_t, a["zp"], a["gp"], a["rows"], a["cols"], a["n"], mp, mn,
              kernel, r_cut, precision, out.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    return out.cpu().numpy()


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("precision,tol", [(0, 1e-10), (1, 2e-6)])
def test_noalloc_matches_workspace_version_twice(cuda, precision, tol):
    from flapjax_b200 import _lib

    mir = (np.array([0.0, -0.2, 0.0]), np.array([0.0, 1.0, 0.0]))
    for call, (seed, shapes, n_t, kernel, mirror) in enumerate([
            (1, [(6, 9), (20, 9)], 500, _lib.FJ_KERNEL_EPSILON, None),
            (2, [(12, 30)], 1500, _lib.FJ_KERNEL_CUTOFF, None),
            (4, [(5, 8), (15, 8)], 700, _lib.FJ_KERNEL_EPSILON, mir)]):
        rng = np.random.default_rng(seed)
        lats = _lattices(rng, shapes)
        targets = rng.normal(size=(n_t, 3)) * [1.0, 2.0, 0.3] + [0.5, 1.5, 0.0]
        a = _args(cuda, targets, lats)
        want = _with_workspace(cuda, a, n_t, kernel, 1e-3, precision, mirror)
        got = _no_alloc(cuda, a, n_t, kernel, 1e-3, precision, mirror)
        assert _rel(got, want) < tol, (call, _rel(got, want))
        kname = "epsilon" if kernel == _lib.FJ_KERNEL_EPSILON else "cutoff"
        ref = R.compute_v_ind(targets, [z for z, _ in lats], [g for _, g in lats], kname, mirror, 1e-3)
        assert _rel(got, ref) < tol, (call, _rel(got, ref))


@pytest.mark.parametrize("precision,tol", [(0, 1e-10), (1, 2e-6)])
def test_noalloc_caps_splits_to_its_array(cuda, precision, tol):
    """20 000 targets against a 60 x 200 lattice: one set of partial velocities is 480 kB,
    so about 14 splits fit beside the filament stream, fewer than the 22 (FP64) or 33
    (FP32) that fj_vind picks; the result must not depend on the split count."""
    from flapjax_b200 import _lib

    rng = np.random.default_rng(9)
    lats = _lattices(rng, [(60, 200)])
    n_t = 20000
    targets = rng.normal(size=(n_t, 3)) * [1.0, 2.0, 0.3] + [0.5, 1.5, 0.0]
    a = _args(cuda, targets, lats)
    got = _no_alloc(cuda, a, n_t, _lib.FJ_KERNEL_EPSILON, 0.0, precision)
    want = _with_workspace(cuda, a, n_t, _lib.FJ_KERNEL_EPSILON, 0.0, precision)
    assert _rel(got, want) < tol
    sub = rng.choice(n_t, 256, replace=False)
    ref = R.compute_v_ind(targets[sub], [lats[0][0]], [lats[0][1]], "epsilon")
    assert _rel(got[sub], ref) < tol


def test_noalloc_refuses_sizes_beyond_its_array(cuda):
    from flapjax_b200 import _lib

    rng = np.random.default_rng(3)
    lats = _lattices(rng, [(400, 200)])  # 2 x 401 x 201 stream elements x 64 B > 8 MiB
    targets = rng.normal(size=(4, 3))
    a = _args(cuda, targets, lats)
    with pytest.raises(_lib.FjError) as e:
        _no_alloc(cuda, a, 4, _lib.FJ_KERNEL_EPSILON, 0.0, _lib.FJ_PREC_FP64)
    assert e.value.code == _lib.FJ_ERR_SHAPE
    assert "fixed" in str(e.value)
