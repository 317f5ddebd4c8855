"""Host-side setup mirrors the reference: geometry, injection, validation. CPU only."""
from dataclasses import replace

import numpy as np
import pytest

from conftest import load_golden
from trench_b200 import geometry, inject
from trench_b200.params import Params


def small(**kw):
    base = dict(nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, bias="dc")
    return replace(Params(), **{**base, **kw})


@pytest.mark.parametrize("name", ["trace_small_barrier", "trace_taper_barrier", "trace_cfg1", "trace_cfg2",
                                  "fields_dielectric"])
def test_geometry_matches_reference(name):
    g = load_golden(f"{name}.npz")
    solid, mask, _, _ = geometry.build_geometry(g["p"])
    np.testing.assert_array_equal(solid, g["solid"])
    if "mask" in g:
        np.testing.assert_array_equal(mask, g["mask"])


@pytest.mark.parametrize("name", ["trace_small_barrier", "trace_cfg1", "trace_cfg2"])
def test_injection_reproduces_reference_particles(name):
    g = load_golden(f"{name}.npz")
    p = g["p"]
    seed = {"trace_small_barrier": 20, "trace_cfg1": 100, "trace_cfg2": 101}[name]
    n = len(g["x"]) // 2
    parts = inject.inject(p, n, g["solid"].shape[1], np.random.default_rng(seed))
    for k, v in zip(("x", "y", "vx", "vy", "qm", "spc"), parts):
        np.testing.assert_array_equal(v, g[k])


@pytest.mark.parametrize("offset", [-6, 0, 6])
def test_shifted_opening(offset):
    """trench tests/test_features.py:23-30"""
    p = small(trench_offset=offset)
    solid, mask, i0, i1 = geometry.build_geometry(p)
    assert i0 == 7 + offset and i1 == 13 + offset
    assert not solid[i0:i1, p.floor_t:].any()
    assert np.array_equal(mask, solid & (np.arange(solid.shape[1])[None, :] >= 16))


@pytest.mark.parametrize("changes", [dict(trench_offset=-7), dict(trench_offset=7), dict(trench_offset=0.5),
                                     dict(trench_taper_deg=90), dict(mask_taper_deg=np.nan),
                                     dict(trench_taper_deg=40), dict(mask_type="metal"), dict(mask_t=-1)])
def test_invalid_geometry_is_rejected(changes):
    with pytest.raises(ValueError):
        geometry.build_geometry(small(**changes))


def test_tapered_openings_match_reference_known_answers():
    """trench tests/test_taper.py:53-69"""
    tr, ma = np.degrees(np.arctan(.25)), np.degrees(np.arctan(.5))
    p = replace(Params(), nx=40, trench_w=16, trench_d=20, floor_t=4, mask_t=12, n_vac=10,
                trench_taper_deg=tr, mask_taper_deg=ma)
    solid, mask, i0, i1 = geometry.build_geometry(p)
    assert (i0, i1) == (12, 28)
    assert geometry.opening_span(solid, p.floor_t) == (17, 23)
    assert geometry.opening_span(solid, p.floor_t + p.trench_d - 1) == (12, 28)
    assert geometry.opening_span(solid, p.floor_t + p.trench_d + p.mask_t - 1) == (6, 34)
    np.testing.assert_array_equal(solid, solid[::-1])


def test_samplers_shapes_and_ranges():
    p = Params()
    rng = np.random.default_rng(0)
    e = inject.mixture_energy([(0.5, "normal", 40, 6), (0.5, "normal", 140, 6)])(rng, 10000)
    assert abs(np.mean(e) - 90) < 1.5
    vx, vy = inject.energy_angle_sampler(p, lambda r, n: np.full(n, 100.0), inject.half_gaussian_angle(3))(rng, 5000)
    assert (vy < 0).all()
    ang = np.degrees(np.arctan2(vx, -vy))
    assert 2.0 < np.std(ang) < 4.0 and abs(np.mean(ang)) < 0.2


def test_sweep_cases_are_valid_and_spread():
    from trench_b200.batch import sweep_params
    ps, seps = sweep_params(64, seed=0)
    assert len(ps) == 64
    for p in ps:
        geometry.build_geometry(p)       # every drawn geometry is valid
        assert 12 <= p.trench_w <= 40 and 40 <= p.trench_d <= 200 and -3 <= p.trench_taper_deg <= 5
        assert 2 ** 15 - 1 <= p.n_per_batch <= 2 ** 17 + 1
    kinds = {p.mask_type for p in ps}
    assert kinds == {"conductor", "dielectric"}
    assert 30 <= min(seps) and max(seps) <= 150


def test_philox_known_answer_vectors():
    """Philox4x32-10 known-answer vectors of the published Random123 test set."""
    from trench_b200.inject import philox4x32_10
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for c, k, want in kat:
        assert tuple(int(v) for v in philox4x32_10([c], k)[0]) == want


def test_histogram_tables():
    from trench_b200.inject import bimodal_gaussian_pdf, histogram_table, table_from_pdf
    e, c = histogram_table([0, 1, 2, 4], [1, 0, 3])
    np.testing.assert_allclose(c, [0, 0.25, 0.25, 1.0])
    with pytest.raises(ValueError):
        histogram_table([0, 1, 1], [1, 1])
    with pytest.raises(ValueError):
        histogram_table([0, 1, 2], [0, 0])
    e, c = table_from_pdf(bimodal_gaussian_pdf(40, 6, 140, 6), 0, 200)
    assert c[0] == 0 and c[-1] == 1 and np.all(np.diff(c) >= 0)
    # the median of the symmetric bimodal density lies between the peaks
    assert 60 < np.interp(0.5, c, e) < 120


@pytest.mark.parametrize("change", [dict(bias="dc"), dict(top_bc="neumann"), dict(rf_time_steps=0),
                                    dict(dt_batch=1e-12)])
def test_invalid_rf_cycle_settings_are_rejected(change):
    """circuit_rf needs the RF bias, a Dirichlet top, at least 16 clock steps per period and
    batches of at least one period (tests/test_rf_cycle.py:159-165)."""
    from trench_b200.fields import field_voltages
    settings = dict(nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, field_mode="circuit_rf",
                    bias="rf", side_bc="pillar", rf_freq=2.5e9, sigma_s=0)
    p = replace(Params(), **{**settings, **change})
    solid, mask, _, _ = geometry.build_geometry(p)
    t = np.arange(256) * 4e-10 / 256
    circuit = dict(t=t, uw=-80 + 0 * t, um=-40 + 0 * t, up=10 + 0 * t, V1=50 + 0 * t)
    with pytest.raises(ValueError):
        field_voltages(p, mask, circuit)


def test_circuit_phase_is_periodic_and_gauge_invariant():
    """tests/test_features.py:97-104: electrode voltages relative to the plasma, periodic in phase."""
    from trench_b200.fields import circuit_voltages
    c = dict(t=np.arange(4) * 1e-8, uw=np.array([-80.0, -100.0, -80.0, -60.0]),
             um=np.array([-40.0, -50.0, -40.0, -30.0]), up=np.full(4, 10.0), V1=np.array([50.0, 60.0, 50.0, 40.0]))
    v = circuit_voltages(c, 45)
    assert v == dict(substrate=-100, mask=-55, top=0, sheath=55)
    assert circuit_voltages(c, 405) == v
    for k in ("uw", "um", "up"):
        c[k] = c[k] + 123
    assert circuit_voltages(c, 45) == v


def _saved_run():
    from dataclasses import asdict
    g = load_golden("run_floating_leak.npz")
    p = g["p"]
    hist = {k[5:]: g[k] for k in g if k.startswith("hist_")}
    return p, dict(params=asdict(p), rho_raw=g["rho_raw"], hist=hist, solid=g["solid"], mask=g["mask"],
                   checkpoint=dict(version=1, batches_completed=len(hist["t"]), steady_n_ok=0))


@pytest.mark.parametrize("changes", [dict(trench_offset=1), dict(dt_batch=2e-4), dict(flux=2e20), dict(rf_volt=200),
                                     dict(n_per_batch=256), dict(seed=2)])
def test_resume_rejects_changes_to_physics_and_particles(changes):
    """tests/test_resume.py:164-170: a resumed run keeps the saved geometry, physics and particles."""
    from trench_b200.step import validate_resume
    p, res = _saved_run()
    with pytest.raises(ValueError, match="keep the geometry"):
        validate_resume(res, replace(p, **changes))


def test_resume_accepts_loop_settings_and_display_rounding():
    from trench_b200.step import validate_resume
    p, res = _saved_run()
    n = len(res["hist"]["t"])
    assert validate_resume(res, replace(p, n_batches=5, steady_rtol=0.01)) == n
    assert validate_resume(res, replace(p, dt_batch=p.dt_batch * (1 + 1e-12), dx=p.dx * (1 - 1e-12))) == n


def test_resume_rejects_invalid_cap_history_and_checkpoint():
    """tests/test_resume.py:181-193."""
    import copy
    from trench_b200.step import validate_resume
    p, res = _saved_run()
    n = len(res["hist"]["t"])
    with pytest.raises(ValueError, match="whole run"):
        validate_resume(res, replace(p, until_steady=True, max_batches=n))
    damaged = copy.deepcopy(res)
    damaged["hist"]["t"] = damaged["hist"]["t"].copy()
    damaged["hist"]["t"][-1] += p.dt_batch
    with pytest.raises(ValueError, match="continuous history"):
        validate_resume(damaged, p)
    damaged = copy.deepcopy(res)
    damaged["checkpoint"]["batches_completed"] = n - 1
    with pytest.raises(ValueError, match="batch count"):
        validate_resume(damaged, p)
    damaged = copy.deepcopy(res)
    damaged["rho_raw"] = damaged["rho_raw"][:-1]
    with pytest.raises(ValueError, match="wrong shape"):
        validate_resume(damaged, p)
