"""Autotuner of the Biot-Savart sum launches (fj_autotune_vind): tuned splits stay within
the workspace bound, the table round-trips, and a case solved with tuned splits gives the
same answer as with the wave-filling rule (1e-12 in FP64, 1e-6 in mixed)."""
from __future__ import annotations

import numpy as np
import pytest

from flapjax_b200 import cases
from tests.helpers import device_uvlm, rel_err

pytestmark = pytest.mark.gpu


def _solve(c, precision):
    uv, _ = device_uvlm(c, precision)
    return uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_tuned_splits_give_the_same_answer(cuda, precision, tol, tmp_path):
    from flapjax_b200 import tuning

    c = cases.wing_free(m=6, n=24, m_star=30, n_steps=4, seed=3)
    tuning.set_table(None)
    want = _solve(c, precision)
    res = tuning.autotune(tuning.step_shapes(c.m, c.n, c.m_star, True), precision=precision)
    for r in res:
        assert r["split"] >= 1 and r["ms"] > 0 and r["rule_ms"] > 0
        assert r["ms"] <= r["rule_ms"] * 1.02 + 1e-6
    t = tuning.table()
    assert np.count_nonzero(t) >= 1
    got = _solve(c, precision)
    for a, b in zip(got.gamma_b, want.gamma_b):
        assert rel_err(a, b) < tol
    # the table survives a save / drop / load round trip
    p = tmp_path / "tune.json"
    tuning.save(p)
    tuning.set_table(None)
    assert np.count_nonzero(tuning.table()) == 0
    tuning.load(p)
    assert np.array_equal(tuning.table(), t)
    tuning.set_table(None)


def test_wide_tile_gives_the_same_answer(cuda):
    """Four targets per thread (the tile the autotuner may pick for an FP32 sum) against
    the default two: a table that asks for the wide tile and 8 splits on every FP32 shape
    reproduces the default run within the mixed tolerance (1e-6), single-case and batched."""
    from flapjax_b200 import tuning
    from flapjax_b200.serving import BatchStepper

    c = cases.wing_free(m=6, n=24, m_star=30, n_steps=4, seed=3)
    tuning.set_table(None)
    want = _solve(c, "mixed")
    t = np.zeros_like(tuning.table())
    half = t.size // 2  # the FP64 block first, then the FP32 block
    t[half:] = 8 | 0x1000
    tuning.set_table(t)
    try:
        got = _solve(c, "mixed")
        uv, _ = device_uvlm(c, "mixed")
        dc = uv.make_device_case(c.n_tstep)
        uv.load_initial(dc, uv.solve_static())
        dc.set_hg(c.hg_t, c.hg_dot_t)
        dc.solve_dynamic(1, 2)
        st = BatchStepper(2, cuda)
        for i in range(2, c.n_tstep):
            st.step([dc], [i], [True])
        batched = uv._to_case(dc)
        st.close()
    finally:
        tuning.set_table(None)
    for case in (got, batched):
        for a, b in zip(case.gamma_b, want.gamma_b):
            assert rel_err(a, b) < 1e-6
