"""The C-ABI library: loads without a GPU, exports every symbol include/fj_uvlm.h
declares, and the ctypes mirrors of its structs have the C layout."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from flapjax_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "fj_uvlm.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^FJ_API\s+[\w\s\*]*?\b(fj_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("fj_vind", "fj_aic_assemble", "fj_lu_factor", "fj_solve_static", "fj_solve_prescribed_dynamic",
                 "fj_case_step", "fj_solve_mixed", "fj_last_error_string"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    if not _lib.LIB_PATH.exists():
        pytest.skip("libfj_uvlm.so not built (run __graft_entry__.build())")
    lib = C.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(_lib.EXPORTED)


def test_error_string_without_gpu():
    lib = _lib.load()
    # a shape error is raised before any CUDA call
    cfg = _lib.FjCaseConfig()
    cfg.n_surf = 0
    nbytes = C.c_size_t()
    st = lib.fj_case_workspace_size(C.byref(cfg), C.byref(nbytes))
    assert st == _lib.FJ_ERR_SHAPE
    assert b"n_surf" in lib.fj_last_error_string()
    with pytest.raises(_lib.FjError):
        _lib.check(st)


def test_influence_jacobian_arguments_are_checked_on_cpu():
    """The linear model's entry points reject bad arguments before any CUDA call."""
    lib = _lib.load()
    buf = (C.c_double * 64)()
    p = C.cast(buf, C.c_void_p)
    # the unregularised kernel has no hand-written derivatives
    st = lib.fj_vertex_jacobian(p, 2, None, p, p, 1, 1, None, None, _lib.FJ_KERNEL_PLAIN, 0.0, p, 12, None)
    assert st == _lib.FJ_ERR_UNSUPPORTED and b"epsilon and cutoff" in lib.fj_last_error_string()
    st = lib.fj_ring_influence(p, 2, None, p, 1, 1, None, None, _lib.FJ_KERNEL_PLAIN, 0.0, p, 1, None)
    assert st == _lib.FJ_ERR_UNSUPPORTED
    # leading dimension below the block width; negative sizes; null outputs
    assert lib.fj_ring_influence(p, 2, None, p, 2, 3, None, None, _lib.FJ_KERNEL_EPSILON, 0.0, p, 5,
                                 None) == _lib.FJ_ERR_SHAPE
    assert lib.fj_vertex_jacobian(p, 2, None, p, p, 1, 1, None, None, _lib.FJ_KERNEL_EPSILON, 0.0, p, 11,
                                  None) == _lib.FJ_ERR_SHAPE
    assert lib.fj_vertex_jacobian(p, -1, None, p, p, 1, 1, None, None, _lib.FJ_KERNEL_EPSILON, 0.0, p, 12,
                                  None) == _lib.FJ_ERR_SHAPE
    assert lib.fj_ring_influence(p, 2, None, p, 1, 1, None, None, _lib.FJ_KERNEL_EPSILON, 0.0, None, 1,
                                 None) == _lib.FJ_ERR_SHAPE
    # the many-right-hand-side solve: workspace, leading dimension
    nb = C.c_size_t()
    assert lib.fj_lu_solve_many_workspace_size(100, 300, C.byref(nb)) == _lib.FJ_OK
    assert nb.value >= 100 * 300 * 8 + 100 * 4
    assert lib.fj_lu_solve_many(p, 100, p, p, 300, 300, p, nb.value - 1, None) == _lib.FJ_ERR_NOMEM
    assert lib.fj_lu_solve_many(p, 100, p, p, 300, 299, p, nb.value, None) == _lib.FJ_ERR_SHAPE
    assert lib.fj_lu_solve_many_workspace_size(0, 3, C.byref(nb)) == _lib.FJ_ERR_SHAPE


def test_workspace_size_is_computable_on_cpu():
    cfg = _lib.FjCaseConfig()
    cfg.n_surf = 1
    cfg.m[0], cfg.n[0], cfg.m_star[0] = 16, 128, 200
    cfg.n_nodes, cfg.n_tstep, cfg.dt = 129, 201, 1.0 / 16
    cfg.kernel = _lib.FJ_KERNEL_CUTOFF
    cfg.r_cut = 1e-3
    cfg.precision = _lib.FJ_PREC_MIXED
    cfg.flow.u_inf[0] = 1.0
    nbytes = C.c_size_t()
    _lib.call("fj_case_workspace_size", C.byref(cfg), C.byref(nbytes))
    nb = 16 * 128
    assert nbytes.value > 2 * nb * nb * 4 + nb * nb * 8  # FP32 factors + inverse + FP64 AIC


def _c_layout():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "fj_uvlm.h"
#define P(T, F) printf(#T "." #F " %zu\n", offsetof(T, F));
int main(void) {
  printf("fj_flowfield %zu\nfj_case_config %zu\nfj_case_buffers %zu\nfj_profile %zu\n",
         sizeof(fj_flowfield), sizeof(fj_case_config), sizeof(fj_case_buffers), sizeof(fj_profile));
  P(fj_case_config, flow) P(fj_case_config, precision) P(fj_case_config, dt) P(fj_case_config, mirror_normal)
  P(fj_flowfield, gust_x0) P(fj_case_buffers, d_force_total) P(fj_profile, vind_pairs)
  P(fj_profile, vind64_pairs)
  return 0;
}
'''
    return src


def test_struct_layouts_match_header(tmp_path):
    exe = tmp_path / "layout"
    (tmp_path / "l.c").write_text(_c_layout())
    r = subprocess.run(["gcc", "-I", str(ROOT / "include"), str(tmp_path / "l.c"), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True,
                                                              text=True).stdout.splitlines())
    assert int(out["fj_flowfield"]) == C.sizeof(_lib.FjFlowfield)
    assert int(out["fj_case_config"]) == C.sizeof(_lib.FjCaseConfig)
    assert int(out["fj_case_buffers"]) == C.sizeof(_lib.FjCaseBuffers)
    assert int(out["fj_profile"]) == C.sizeof(_lib.FjProfile)
    assert int(out["fj_case_config.flow"]) == _lib.FjCaseConfig.flow.offset
    assert int(out["fj_case_config.precision"]) == _lib.FjCaseConfig.precision.offset
    assert int(out["fj_case_config.dt"]) == _lib.FjCaseConfig.dt.offset
    assert int(out["fj_case_config.mirror_normal"]) == _lib.FjCaseConfig.mirror_normal.offset
    assert int(out["fj_flowfield.gust_x0"]) == _lib.FjFlowfield.gust_x0.offset
    assert int(out["fj_case_buffers.d_force_total"]) == _lib.FjCaseBuffers.d_force_total.offset
    assert int(out["fj_profile.vind_pairs"]) == _lib.FjProfile.vind_pairs.offset
    assert int(out["fj_profile.vind64_pairs"]) == _lib.FjProfile.vind64_pairs.offset


def test_autograd_module_imports_without_a_gpu():
    from flapjax_b200 import autograd

    assert callable(autograd.induced_velocity) and callable(autograd.dense_solve)


def test_tuning_shapes_of_a_step():
    from flapjax_b200 import tuning

    s = tuning.step_shapes(16, 128, 200, True)
    assert s[0] == (16 * 128, 2 * 201 * 129)
    assert s[1] == (16 * 129 + 17 * 128, 2 * 17 * 129 + 2 * 201 * 129)
    assert s[2] == (201 * 129, 2 * 17 * 129 + 2 * 201 * 129)
    assert len(tuning.step_shapes(4, 8, 10, False)) == 2


def test_jax_binding_is_import_guarded():
    """flapjax_b200.fj_jax (the jax.ffi / custom_vjp binding) imports without JAX, reports
    itself unavailable and refuses to register; its handler source names only exported
    entry points."""
    import re

    from flapjax_b200 import build, fj_jax

    if fj_jax.jax is None:
        assert not fj_jax.available()
        with pytest.raises(RuntimeError, match="needs JAX"):
            fj_jax.register()
        assert build.xla_include_dir() is None
    src = (ROOT / "flapjax_b200" / "xla" / "fj_xla.cc").read_text()
    header = (ROOT / "include" / "fj_uvlm.h").read_text()
    for name in set(re.findall(r"\b(fj_[a-z0-9_]+)\(", src)):
        assert f"FJ_API int {name}(" in header or f"FJ_API const char* {name}(" in header, name
    for sym in fj_jax._TARGETS.values():
        assert f"XLA_FFI_DEFINE_HANDLER_SYMBOL({sym}," in src


def test_autotune_table_accepts_tiles_only_for_fp32():
    """A tuned table entry is a split count (1..1024), plus 4096 for the four-target tile
    in the FP32 half only; fj_autotune_set checks that on the host, with no GPU."""
    import numpy as np

    from flapjax_b200 import tuning

    n = C.c_int()
    _lib.call("fj_autotune_table_size", C.byref(n))
    t = np.zeros(n.value, dtype=np.int16)
    t[n.value // 2] = 8 | 0x1000
    tuning.set_table(t)
    assert tuning.table()[n.value // 2] == 8 | 0x1000
    for bad_at, bad in ((0, 8 | 0x1000), (1, 1025), (n.value - 1, 0x1000)):
        b = np.zeros_like(t)
        b[bad_at] = bad
        with pytest.raises(_lib.FjError):
            tuning.set_table(b)
    tuning.set_table(None)
