"""Steady-state stopping: the check functions against the reference's outputs on
seeded synthetic histories (trench_charging_2d.py:877-945)."""
import numpy as np
import pytest

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


def _p(**changes):
    from dataclasses import replace
    from trench_b200.params import Params
    return replace(Params(), steady_window=30, **changes)


@pytest.mark.parametrize("sign", [-1, 1])
@pytest.mark.parametrize("age", [10_000, 1_000_000])
def test_constant_charging_fails_the_drift_check_although_the_means_are_close(sign, age):
    """A steady current passes the relative block-mean test after a long run but not the drift
    test (tests/test_steady_charge.py:17-28)."""
    p = _p()
    W = p.steady_window
    q = sign * (age + np.arange(2 * W)) * 1e-12
    cur, prev = q[-W:].mean(), q[:W].mean()
    assert abs(cur - prev) < p.steady_charge_rtol * max(abs(cur), abs(prev))
    check = steady.check_charge_steady({"right": q}, p)
    assert not check["ok"] and check["kind"] == "drift"
    np.testing.assert_allclose(check["d"], sign * W * 1e-12, rtol=1e-8)
    np.testing.assert_allclose(check["rate"], sign * 1e-12 / p.dt_batch, rtol=1e-8)


@pytest.mark.parametrize("seed", [3, 17])
def test_stationary_charge_with_sampling_noise_passes(seed):
    p = _p()
    noise = np.random.default_rng(seed).normal(0, 0.01e-12, 2 * p.steady_window)
    assert steady.check_charge_steady({"left": 20e-12 + noise, "right": -50e-12 - noise}, p)["ok"]


def test_a_recent_step_fails_the_block_mean_check():
    p = _p()
    q = np.r_[np.full(p.steady_window, 20e-12), np.full(p.steady_window, 21e-12)]
    check = steady.check_charge_steady({"bottom": q}, p)
    assert not check["ok"] and check["kind"] == "mean"
    np.testing.assert_allclose(check["d"], 1e-12)


def test_opposite_walls_and_the_absolute_surface_charge_are_checked_separately():
    p = _p()
    q = (100 + np.arange(2 * p.steady_window) * 0.05) * 1e-12
    check = steady.check_charge_steady({"left": q, "right": -q, "surface": q - q}, p)
    assert not check["ok"] and check["name"] in ("left", "right")
    g = np.arange(2 * p.steady_window) * 1e-12
    check = steady.check_charge_steady({"surface": np.zeros_like(g), "surface absolute": g}, p)
    assert not check["ok"] and check["name"] == "surface absolute"


def test_negligible_drift_uses_the_absolute_tolerance():
    from dataclasses import replace
    p = _p()
    q = np.arange(2 * p.steady_window) * (p.steady_charge_atol / (2 * p.steady_window))
    assert steady.check_charge_steady({"left": q}, p)["ok"]
    assert steady.check_charge_steady({"left": np.zeros_like(q)}, replace(p, steady_charge_atol=0))["ok"]


@pytest.mark.parametrize("changes", [dict(steady_charge_rtol=0), dict(steady_charge_rtol=np.nan),
                                     dict(steady_charge_atol=-1), dict(steady_charge_atol=np.inf),
                                     dict(steady_window=4), dict(dt_batch=0)])
def test_invalid_charge_criterion_is_rejected(changes):
    from dataclasses import replace
    with pytest.raises(ValueError):
        steady.check_charge_steady({"left": np.zeros(60)}, replace(_p(), **changes))


@pytest.mark.parametrize("mask_type", ["conductor", "dielectric"])
def test_charge_monitors_cover_both_walls_height_bands_floor_and_mask(mask_type):
    """tests/test_steady_charge.py:77-99: the monitor regions of the charge check."""
    from dataclasses import replace
    from trench_b200 import geometry
    from trench_b200.params import Params
    p = replace(Params(), nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, mask_type=mask_type)
    solid, mask, i0, i1 = geometry.build_geometry(p)
    regions = steady.charge_monitors(solid, mask, i0, i1, p)
    rho = np.zeros(solid.shape)
    rho[i0 - 1, p.floor_t + 1] = 3 / p.dx ** 2
    rho[i0 - 1, p.floor_t + p.trench_d - 1] = -3 / p.dx ** 2
    rho[i1, p.floor_t + 1] = 2 / p.dx ** 2
    rho[i0 + 1, p.floor_t - 1] = 5 / p.dx ** 2
    rho.flat[np.flatnonzero(mask & geometry.surface_cells(solid))[0]] = 7 / p.dx ** 2
    q = {k: rho.ravel()[idx].sum() * p.dx ** 2 for k, idx in regions.items()}
    absolute = np.abs(rho.ravel()[regions["surface"]]).sum() * p.dx ** 2
    np.testing.assert_allclose([q["left"], q["left band 1"], q["left band 3"], q["right"], q["bottom"], q["mask"]],
                               [0, 3, -3, 2, 5, 7], atol=1e-12)
    np.testing.assert_allclose(q["surface"], 7 if mask_type == "conductor" else 14)
    np.testing.assert_allclose(absolute, 13 if mask_type == "conductor" else 20)
