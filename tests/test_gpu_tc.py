"""Tensor-core products (fj_gemm_tf32) and the tensor-core factorisation behind the mixed
solve (jnp.linalg.solve, aero/uvlm.py:985).

The GEMM is checked elementwise against the FP64 product, with error bounds scaled by
|A| |B|: three-pass split within 1e-5 (FP32-class), one TF32 pass within 3e-3.  The mixed
solve must reach the same refined answer whichever factor path made its inverse.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def _f32(a, dev):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(dev)


def _call_gemm(cuda, kernel, pa, lda, pb, ldb, pc, ldc, m, n, k, alpha, beta, passes, err):
    """One product through fj_gemm_tf32 (kernel "staged") or fj_gemm_tf32_tma ("tma",
    with its operand-split scratch)."""
    import torch

    from flapjax_b200 import _lib

    s = torch.cuda.current_stream(cuda).cuda_stream
    if kernel == "staged":
        _lib.call("fj_gemm_tf32", pa, lda, pb, ldb, pc, ldc, m, n, k, C.c_float(alpha), C.c_float(beta), passes,
                  err.data_ptr(), s)
        return
    nf = C.c_size_t()
    _lib.call("fj_gemm_tf32_scratch_floats", m, n, k, passes, C.byref(nf))
    scratch = torch.full((nf.value + 4,), float("nan"), dtype=torch.float32, device=cuda)
    _lib.call("fj_gemm_tf32_tma", pa, lda, pb, ldb, pc, ldc, m, n, k, C.c_float(alpha), C.c_float(beta), passes,
              scratch.data_ptr(), nf.value, err.data_ptr(), s)
    torch.cuda.synchronize(cuda)


def _gemm(cuda, a, b, c, m, n, k, alpha, beta, passes, kernel="staged"):
    """C <- alpha A B + beta C on the device; a, b, c are 2-D float32 host arrays whose
    leading (m x k), (k x n), (m x n) blocks are the operands (row strides = their widths)."""
    import torch

    ta, tb, tc = _f32(a, cuda), _f32(b, cuda), _f32(c, cuda)
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    _call_gemm(cuda, kernel, ta.data_ptr(), a.shape[1], tb.data_ptr(), b.shape[1], tc.data_ptr(), c.shape[1], m, n,
               k, alpha, beta, passes, err)
    out = tc.cpu().numpy()
    assert int(err.cpu()) == 0
    return out


@pytest.mark.parametrize("m,n,k,lda,ldb,ldc", [(128, 128, 32, 32, 128, 128), (200, 300, 100, 103, 301, 305),
                                               (5, 7, 3, 3, 7, 7), (384, 256, 128, 131, 257, 256)])
@pytest.mark.parametrize("passes", [1, 3])
@pytest.mark.parametrize("kernel", ["staged", "tma"])
def test_gemm_matches_fp64_product(cuda, m, n, k, lda, ldb, ldc, passes, kernel):
    rng = np.random.default_rng(m + n + k + passes)
    a = rng.normal(size=(m, lda)).astype(np.float32)
    b = rng.normal(size=(k, ldb)).astype(np.float32)
    c = rng.normal(size=(m, ldc)).astype(np.float32)
    alpha, beta = -1.0, 1.0
    got = _gemm(cuda, a, b, c, m, n, k, alpha, beta, passes, kernel)
    A, B = a[:, :k].astype(np.float64), b[:, :n].astype(np.float64)
    want = alpha * A @ B + beta * c[:, :n].astype(np.float64)
    scale = np.abs(A) @ np.abs(B) + np.abs(c[:, :n])
    tol = 1e-5 if passes == 3 else 3e-3
    assert np.all(np.abs(got[:, :n] - want) <= tol * scale)
    # columns past n and the padding of every row stay untouched
    assert np.array_equal(got[:, n:], c[:, n:])


@pytest.mark.parametrize("kernel", ["staged", "tma"])
def test_gemm_split_beats_single_pass_and_beta_zero_ignores_c(cuda, kernel):
    rng = np.random.default_rng(9)
    m, n, k = 256, 256, 128
    a = rng.normal(size=(m, k)).astype(np.float32)
    b = rng.normal(size=(k, n)).astype(np.float32)
    c = np.full((m, n), np.nan, np.float32)  # beta = 0 must not read C
    want = a.astype(np.float64) @ b.astype(np.float64)
    e1 = rel_err(_gemm(cuda, a, b, c, m, n, k, 1.0, 0.0, 1, kernel), want)
    e3 = rel_err(_gemm(cuda, a, b, c, m, n, k, 1.0, 0.0, 3, kernel), want)
    assert e3 < 5e-6 and 100 * e3 < e1 < 1e-2


@pytest.mark.parametrize("kernel", ["staged", "tma"])
def test_gemm_in_place_on_b(cuda, kernel):
    """U12 = L11^-1 A12 runs in place (C is B's memory, m <= 128)."""
    import torch

    rng = np.random.default_rng(3)
    m = k = 128
    n = 500
    a = rng.normal(size=(m, k)).astype(np.float32)
    b = rng.normal(size=(k, n)).astype(np.float32)
    ta, tb = _f32(a, cuda), _f32(b, cuda)
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    _call_gemm(cuda, kernel, ta.data_ptr(), k, tb.data_ptr(), n, tb.data_ptr(), n, m, n, k, 1.0, 0.0, 3, err)
    want = a.astype(np.float64) @ b.astype(np.float64)
    assert rel_err(tb.cpu().numpy(), want) < 5e-6
    assert int(err.cpu()) == 0


def test_gemm_tma_overlapping_update(cuda):
    """A22 -= A21 A12 inside one matrix (the trailing update's aliasing: A and B are
    blocks of C's own matrix), several K slabs, ragged edges."""
    import torch

    rng = np.random.default_rng(11)
    n, k0 = 700, 160
    a = rng.normal(size=(n, n)).astype(np.float32)
    ta = _f32(a, cuda)
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    base, es = ta.data_ptr(), 4
    rest = n - k0
    _call_gemm(cuda, "tma", base + k0 * n * es, n, base + k0 * es, n, base + (k0 * n + k0) * es, n, rest, rest, k0,
               -1.0, 1.0, 3, err)
    A = a.astype(np.float64)
    want = A.copy()
    want[k0:, k0:] -= A[k0:, :k0] @ A[:k0, k0:]
    got = ta.cpu().numpy()
    scale = np.abs(A[k0:, :k0]) @ np.abs(A[:k0, k0:]) + np.abs(A[k0:, k0:])
    assert np.all(np.abs(got[k0:, k0:] - want[k0:, k0:]) <= 1e-5 * scale)
    assert np.array_equal(got[:k0], a[:k0]) and np.array_equal(got[:, :k0], a[:, :k0])
    assert int(err.cpu()) == 0


def _solve_mixed(cuda, a, b):
    import torch

    from flapjax_b200 import _lib

    n = a.shape[0]
    nbytes = C.c_size_t()
    _lib.call("fj_solve_mixed_workspace_size", n, C.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=cuda)
    ta = torch.as_tensor(a).to(cuda)
    tb = torch.as_tensor(b).to(cuda)
    tx = torch.empty(n, dtype=torch.float64, device=cuda)
    res = torch.empty(1, dtype=torch.float64, device=cuda)
    s = torch.cuda.current_stream(cuda).cuda_stream
    _lib.call("fj_solve_mixed", ta.data_ptr(), n, tb.data_ptr(), tx.data_ptr(), 1, res.data_ptr(), ws.data_ptr(),
              ws.numel(), s)
    return tx.cpu().numpy(), float(res.cpu())


@pytest.mark.parametrize("n", [256, 300, 777, 1500])
def test_mixed_solve_through_tensor_core_factors(cuda, n, monkeypatch):
    rng = np.random.default_rng(n)
    a = rng.normal(size=(n, n)) + n * 0.05 * np.eye(n)
    b = rng.normal(size=n)
    want = np.linalg.solve(a, b)
    monkeypatch.setenv("FJ_MIXED_FACTOR", "tf32x3")
    x3, r3 = _solve_mixed(cuda, a, b)
    assert r3 < 1e-12 and rel_err(x3, want) < 1e-11
    monkeypatch.setenv("FJ_MIXED_FACTOR", "cuda")
    xc, rc = _solve_mixed(cuda, a, b)
    assert rc < 1e-12 and rel_err(xc, want) < 1e-11
    # one TF32 pass: a coarser inverse, so three refinement sweeps leave more behind
    monkeypatch.setenv("FJ_MIXED_FACTOR", "tf32")
    x1, r1 = _solve_mixed(cuda, a, b)
    assert r1 < 1e-2


@pytest.mark.parametrize("n", [300, 520, 1100, 2200])
def test_mixed_solve_heavy_pivoting(cuda, n, monkeypatch):
    """No diagonal dominance: pivot rows come from far below the outer panel, so the row
    swaps must reach the columns to its right before their updates.  Such a matrix
    (condition number ~1e3) converges more slowly in three refinement sweeps; the
    tensor-core inverse must do as well as the FP32 CUDA-core one."""
    rng = np.random.default_rng(100 + n)
    a = rng.normal(size=(n, n))
    b = rng.normal(size=n)
    want = np.linalg.solve(a, b)
    monkeypatch.setenv("FJ_MIXED_FACTOR", "cuda")
    xc, rc = _solve_mixed(cuda, a, b)
    monkeypatch.setenv("FJ_MIXED_FACTOR", "tf32x3")
    x, r = _solve_mixed(cuda, a, b)
    assert r < max(1e-12, 10 * rc) and rel_err(x, want) < 1e-8 and rel_err(xc, want) < 1e-8


@pytest.mark.parametrize("n", [640, 1029])
def test_mixed_solve_pivot_ties(cuda, n, monkeypatch):
    """Entries of +-1 (and a few exact zeros): the first columns' pivot searches meet
    equal magnitudes everywhere, and the first maximum (the lowest row) must win in the
    cluster-wide search as in getrf.  n = 1029 also leaves a ragged last outer panel and
    rows that start off 16-byte boundaries."""
    rng = np.random.default_rng(7 + n)
    a = rng.choice([-1.0, 1.0], size=(n, n))
    a[rng.random(size=(n, n)) < 0.01] = 0.0
    b = rng.normal(size=n)
    want = np.linalg.solve(a, b)
    monkeypatch.setenv("FJ_MIXED_FACTOR", "cuda")
    xc, rc = _solve_mixed(cuda, a, b)
    monkeypatch.setenv("FJ_MIXED_FACTOR", "tf32x3")
    x, r = _solve_mixed(cuda, a, b)
    assert np.isfinite(r) and r < max(1e-12, 10 * rc)
    assert rel_err(x, want) < max(1e-8, 10 * rel_err(xc, want))


def test_mixed_solve_of_an_aic(cuda):
    """The static AIC of a 16 x 32 wing with a 20-row wake (n = 512): tensor-core factors
    through the refinement to the FP64 solution."""
    from oracle import uvlm_ref as R

    m, n = 16, 32
    z = np.zeros((m + 1, n + 1, 3))
    z[..., 0] = np.linspace(-0.25, 0.75, m + 1)[:, None]
    z[..., 1] = np.linspace(0.0, 8.0, n + 1)[None, :]
    z[..., 2] = 0.05 * z[..., 0] ** 2  # a little camber
    zw = z[-1][None] + np.arange(21)[:, None, None] * np.array([0.125, 0.0, 0.0])  # a straight static wake
    cs, ns = [R.compute_surf_c(z)], [R.compute_surf_nc(z)]
    a = R.compute_aic_solve(cs, ns, [z], [zw], R.KERNEL_EPSILON, None)
    b = np.random.default_rng(0).normal(size=a.shape[0])
    want = np.linalg.solve(a, b)
    x, r = _solve_mixed(cuda, a, b)
    assert r < 1e-12 and rel_err(x, want) < 1e-10


def test_bounded_wait_expires_and_context_survives(cuda):
    """Failure detection without a fault: the GEMM kernel with its MMAs withheld waits on
    an mbarrier that nothing completes; the bounded wait gives up (about 2 s), the kernel
    reports it in the status word and returns, and the next product is correct."""
    import time

    import torch

    from flapjax_b200 import _lib

    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    scratch = torch.zeros(4, dtype=torch.float32, device=cuda)
    s = torch.cuda.current_stream(cuda).cuda_stream
    t0 = time.perf_counter()
    _lib.call("fj_tc_wait_selftest", err.data_ptr(), scratch.data_ptr(), s)
    torch.cuda.synchronize()
    assert int(err.cpu()) == 1
    assert time.perf_counter() - t0 < 30.0
    rng = np.random.default_rng(1)
    a = rng.normal(size=(64, 32)).astype(np.float32)
    b = rng.normal(size=(32, 48)).astype(np.float32)
    got = _gemm(cuda, a, b, np.zeros((64, 48), np.float32), 64, 48, 32, 1.0, 0.0, 3)
    assert rel_err(got, a.astype(np.float64) @ b.astype(np.float64)) < 5e-6


@pytest.mark.parametrize("n", [3200, 6144])
def test_largest_orders_factor(cuda, n):
    """AIC orders up to the validated 6144: the FP64 LU (panel width 8, 4 or 2 by order)
    and the mixed solve (inner panels 16 or 8) both factor and solve."""
    import torch

    from flapjax_b200 import _lib

    rng = np.random.default_rng(n)
    a = rng.normal(size=(n, n)) + n * 0.05 * np.eye(n)
    b = rng.normal(size=n)
    want = np.linalg.solve(a, b)
    ta = torch.as_tensor(a).to(cuda)
    piv = torch.empty(n, dtype=torch.int32, device=cuda)
    nb_ = C.c_size_t()
    _lib.call("fj_lu_workspace_size", n, C.byref(nb_))
    ws = torch.empty(nb_.value, dtype=torch.uint8, device=cuda)
    s = torch.cuda.current_stream(cuda).cuda_stream
    _lib.call("fj_lu_factor", ta.data_ptr(), n, piv.data_ptr(), ws.data_ptr(), ws.numel(), s)
    tb = torch.as_tensor(b).to(cuda)
    _lib.call("fj_lu_solve", ta.data_ptr(), n, piv.data_ptr(), tb.data_ptr(), ws.data_ptr(), ws.numel(), s)
    assert rel_err(tb.cpu().numpy(), want) < 1e-10
    x, r = _solve_mixed(cuda, a, b)
    assert r < 1e-12 and rel_err(x, want) < 1e-11


def test_largest_wing_solves(cuda):
    """A 16 x 384 wing (AIC order 6144, the largest accepted): static and dynamic steps in
    FP64 and mixed agree."""
    from flapjax_b200 import cases
    from tests.helpers import device_uvlm

    c = cases.wing_heave(m=16, n=384, m_star=4, n_steps=2, span=24.0)
    out = {}
    for prec in ("fp64", "mixed"):
        uv, _ = device_uvlm(c, prec)
        out[prec] = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    for i in range(c.n_tstep):
        assert rel_err(out["mixed"].gamma_b[0][i], out["fp64"].gamma_b[0][i]) < 1e-5
