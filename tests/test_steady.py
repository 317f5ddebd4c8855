"""Steady-state stopping: the check functions against the reference's outputs on
seeded synthetic histories (trench_charging_2d.py:877-945)."""
import numpy as np

from conftest import load_golden
from trench_b200 import steady


def test_mean_and_se_matches_reference():
    g = load_golden("steady_checks.npz")
    got = np.array([steady.mean_and_se(x) for x in g["series"]])
    np.testing.assert_allclose(got, g["mean_se"], rtol=1e-12, atol=0)


def test_potential_check_matches_reference():
    g = load_golden("steady_checks.npz")
    p = g["p"]
    names = ["a", "b", "c"]
    outcomes = set()
    for h, want in zip(g["v_hist"], g["v_out"]):
        ok, name, d, tol = steady.check_steady({k: list(v) for k, v in zip(names, h)}, names, p, None)
        assert float(ok) == want[0] and names.index(name) == int(want[1])
        np.testing.assert_allclose([d, tol], want[2:], rtol=1e-12)
        outcomes.add(bool(ok))
    assert outcomes == {True, False}   # the cases cover both answers


def test_charge_check_matches_reference():
    g = load_golden("steady_checks.npz")
    p = g["p"]
    outcomes = set()
    for (left, right), want in zip(g["q_hist"], g["q_out"]):
        c = steady.check_charge_steady({"left": list(left), "right": list(right)}, p)
        assert float(c["ok"]) == want[0]
        assert ["left", "right"].index(c["name"]) == int(want[1]) and float(c["kind"] == "drift") == want[2]
        np.testing.assert_allclose([c["d"], c["tol"], c["ratio"], c["rate"]], want[3:], rtol=1e-12)
        outcomes.add(c["ok"])
    assert outcomes == {True, False}


def test_history_start_skips_missing_values():
    hist = {"a": np.array([np.nan, 1.0, 2.0, 3.0])}
    mon = {"left": np.array([1.0, np.nan, 2.0, 3.0])}
    assert steady.history_start(hist, ["a"], mon) == 2
    assert steady.history_start({"a": np.ones(3)}, ["a"], {"left": np.ones(3)}) == 0


def test_potential_scale_is_the_charging_potential_not_the_rf_bias():
    """Under the RF circuit the potentials are compared relative to the external ones, so a
    large bias does not widen the tolerance (tests/test_rf_cycle.py:148-156)."""
    from dataclasses import replace
    from trench_b200.params import Params
    p = replace(Params(), steady_window=30)
    charging = np.arange(60) * 0.1
    hist = {"wall": charging - 1000}
    assert steady.check_steady(hist, ["wall"], p)[0]          # the bias alone would pass it
    correct = steady.check_steady(hist, ["wall"], p, dict(wall=-1000))
    no_bias = steady.check_steady({"wall": charging}, ["wall"], p, dict(wall=0))
    assert not correct[0]
    np.testing.assert_allclose(correct[2:], no_bias[2:], rtol=1e-12)
