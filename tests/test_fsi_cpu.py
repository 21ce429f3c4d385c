"""The AeroCase surface the reference's fluid-structure and coupled-adjoint callers use,
checked on the CPU against the reference's own results (tests/golden/fsi/*.npz, made by
tests/golden/make_golden.py with the reference's AeroCase): get_states (AeroStates, ravel
order gamma_b, gamma_w, gamma_b_dot, zeta_w), gamma_full, zeta_full and
project_forcing_to_beam with and without the unsteady forces (aero/data_structures.py:
240-298, 464-492; aero/utils.py:666-697)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from flapjax_b200.data_structures import AeroCase, AeroStates, ArrayList, ArrayListShape, project_forcing_to_beam

GOLD = Path(__file__).resolve().parent / "golden" / "fsi"
FIELDS = ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
          "f_unsteady", "alpha")


def _case(d):
    f = {k: [d[f"dyn_{k}"]] for k in FIELDS}
    f["n"] = f.pop("nc")
    n = int(d["dims"][1])
    return AeroCase(**f, t=d["dyn_t"], i_ts=np.arange(d["dyn_t"].size), dof_mapping=[np.arange(n + 1)])


@pytest.mark.parametrize("name", ["fsi_heave", "fsi_free_cutoff"])
def test_case_methods_match_reference(name):
    d = np.load(GOLD / f"{name}.npz")
    case = _case(d)
    slot = int(d["states_slot"])
    st = case.get_states(slot)
    assert isinstance(st, AeroStates)
    assert np.array_equal(st.ravel(), d["states_ravel"])
    assert st.n_states == d["states_ravel"].size
    assert np.array_equal(np.concatenate([np.ravel(g) for g in case.gamma_full(slot)]), d["gamma_full"])
    assert np.array_equal(np.concatenate([np.ravel(z) for z in case.zeta_full(slot)]), d["zeta_full"])
    x0 = [d["zeta_b0"]]
    for key, unsteady in (("proj_unsteady", True), ("proj_steady", False)):
        got = case.project_forcing_to_beam(slot, d["proj_rmat"], x0, unsteady)
        assert np.allclose(got, d[key], rtol=0, atol=1e-13 * np.abs(d[key]).max()), key


def test_states_round_trip_and_snapshot_writes():
    d = np.load(GOLD / "fsi_heave.npz")
    case = _case(d)
    st = case.get_states(2)
    back = AeroStates.from_vector(st.ravel(), st.shapes())
    for k in ("gamma_b", "gamma_w", "gamma_b_dot", "zeta_w"):
        assert all(np.array_equal(a, b) for a, b in zip(getattr(back, k), getattr(st, k)))
    with pytest.raises(ValueError):
        AeroStates.from_vector(st.ravel()[:-1], st.shapes())
    # __setitem__ writes a snapshot's fields into a slot; c and nc stay as they were
    snap = case[4]
    c_before = case.c[0][1].copy()
    case[1] = snap
    for k in ("zeta_b", "gamma_b", "gamma_w", "f_steady", "f_unsteady", "alpha", "zeta_w", "gamma_b_dot"):
        assert np.array_equal(getattr(case, k)[0][1], getattr(snap, k)[0]), k
    assert np.array_equal(case.c[0][1], c_before)
    assert case.t[1] == snap.t
    with pytest.raises(TypeError):
        snap[0] = snap
    with pytest.raises(ValueError):
        case.get_states()


def test_arraylist_is_elementwise():
    a = ArrayList([np.ones((2, 3)), np.arange(4.0)])
    b = ArrayList([2 * np.ones((2, 3)), np.ones(4)])
    s = a + b
    assert len(s) == 2 and np.array_equal(s[0], 3 * np.ones((2, 3))) and np.array_equal(s[1], np.arange(4.0) + 1)
    assert np.array_equal((a * 2.0)[1], 2 * np.arange(4.0))
    assert np.array_equal((2.0 * a)[1], 2 * np.arange(4.0))
    assert a.shape == ArrayListShape([(2, 3), (4,)])
    assert a.size == 10
    assert np.array_equal(ArrayList.from_vector(a.ravel(), a.shape)[0], a[0])
    assert len(a.combine(b)) == 4
    a += b
    assert np.array_equal(a[1], np.arange(4.0) + 1)


def test_projection_sums_columns_and_moments():
    """Hand check of project_forcing_to_beam on one surface: column sums and (R x0) x f."""
    rng = np.random.default_rng(0)
    f = rng.normal(size=(3, 4, 3))
    x0 = rng.normal(size=(3, 4, 3))
    rmat = np.stack([np.eye(3)] * 5)
    out = project_forcing_to_beam([f], rmat, [np.array([0, 1, 2, 4])], [x0])
    assert np.allclose(out[[0, 1, 2, 4], :3], f.sum(axis=0))
    assert np.allclose(out[[0, 1, 2, 4], 3:], np.cross(x0, f).sum(axis=0))
    assert np.all(out[3] == 0.0)
