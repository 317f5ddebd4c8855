"""Vertical-ion probe on the B200 tracer against the reference's probe_vertical_ions
(golden fixtures) and its known answers (tests/test_taper.py:132-157,
tests/test_features.py:135-163)."""
from dataclasses import asdict, replace

import numpy as np
import pytest

from conftest import load_golden
from trench_b200 import geometry
from trench_b200.params import Params

pytestmark = pytest.mark.gpu


def result_of(g):
    p = g["p"]
    return dict(params=asdict(p), solid=g["solid"], mask=g["mask"], rho_raw=g["rho_raw"], t_conv=1e-3,
                stopped=False, circuit=None)


@pytest.mark.parametrize("name", ["taper_empty", "small_charged"])
def test_probe_matches_reference(cuda_device, name):
    from trench_b200.probe import probe_vertical_ions
    g = load_golden(f"probe_{name}.npz")
    res = result_of(g)
    before = res["rho_raw"].copy()
    out = probe_vertical_ions(res, log=None, device=cuda_device)
    np.testing.assert_array_equal(res["rho_raw"], before)   # the probe never changes the charge
    for label in ("charged", "uncharged"):
        r = out[label]
        for k in ("hits", "status", "hit_cells"):
            np.testing.assert_array_equal(r[k], g[f"{label}_{k}"])
        np.testing.assert_array_equal([r["bottom_fraction"], r["escaped"], r["lost"]], g[f"{label}_scalars"])
        for k in ("endpoints", "final_velocity"):
            np.testing.assert_allclose(r[k], g[f"{label}_{k}"], rtol=1e-10, atol=1e-15)
        np.testing.assert_allclose(r["angle_deg"], g[f"{label}_angle_deg"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(r["impact_energy_eV"], g[f"{label}_impact_energy_eV"], rtol=1e-10)
        np.testing.assert_allclose(r["bottom_flux"], g[f"{label}_bottom_flux"], rtol=1e-12)
        np.testing.assert_allclose(r["phi"], g[f"{label}_phi"], rtol=0, atol=1e-9)
        np.testing.assert_array_equal([len(v) for v in r["paths"]], g[f"{label}_path_lengths"])
        np.testing.assert_allclose(np.concatenate(r["paths"]), g[f"{label}_paths"], rtol=1e-10, atol=1e-15)


def test_probe_vertical_and_uncharged_beam_reaches_the_bottom(cuda_device):
    """tests/test_features.py:135-150: exactly vertical ions stay vertical."""
    from trench_b200.probe import probe_vertical_ions
    p = replace(Params(), nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, bias="dc", sigma_s=0,
                probe_ions=120, probe_trajectories=8, max_steps=800)
    solid, mask, _, _ = geometry.build_geometry(p)
    res = dict(params=asdict(p), solid=solid, mask=mask, rho_raw=np.zeros(solid.shape), t_conv=1e-3, stopped=False)
    out = probe_vertical_ions(res, log=None, device=cuda_device)
    for label in ("charged", "uncharged"):
        d = out[label]
        assert d["bottom_fraction"] == 1 and d["lost"] == 0 and d["escaped"] == 0
        assert len(d["paths"]) == p.probe_trajectories
        for pts in d["paths"]:
            np.testing.assert_array_equal(pts[:, 0], np.full(len(pts), pts[0, 0]))
            np.testing.assert_allclose(pts[-1, 1], p.floor_t * p.dx, atol=1e-18)
        np.testing.assert_array_equal(d["angle_deg"], np.zeros(p.probe_ions))


def test_probe_requires_a_steady_result(cuda_device):
    import threading
    from trench_b200.probe import probe_vertical_ions
    p = replace(Params(), nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, bias="dc", sigma_s=0,
                probe_ions=50, probe_trajectories=5)
    solid, mask, _, _ = geometry.build_geometry(p)
    res = dict(params=asdict(p), solid=solid, mask=mask, rho_raw=np.zeros(solid.shape), t_conv=np.nan)
    with pytest.raises(ValueError):
        probe_vertical_ions(res, log=None, device=cuda_device)
    res["t_conv"] = 1e-3
    stop = threading.Event()
    stop.set()
    assert probe_vertical_ions(res, log=None, stop=stop, device=cuda_device)["cancelled"]


def test_full_cycle_probe_uses_identical_phases_and_preserves_charge(cuda_device):
    """circuit_rf probe (tests/test_rf_cycle.py:176-193, without the plots): the charged and
    uncharged beams start at the same stratified phases, the clock runs in flight, the
    charge is untouched and every ion is accounted for."""
    from trench_b200.probe import probe_vertical_ions
    p = replace(Params(), nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, field_mode="circuit_rf",
                bias="rf", side_bc="pillar", rf_freq=2.5e9, sigma_s=0, probe_ions=128, probe_trajectories=8,
                max_steps=1000, probe_energy_eV=1.5)
    period = 4e-10
    t = np.arange(256) * period / 256
    up = 10 + 2 * np.cos(2 * np.pi * t / period)
    circuit = dict(t=t, up=up, uw=-80 - 35 * np.sin(2 * np.pi * t / period) + up,
                   um=-40 - 17.5 * np.sin(2 * np.pi * t / period) + up, V1=50 + 0 * t)
    solid, mask, i0, _ = geometry.build_geometry(p)
    rho = np.zeros(solid.shape)
    rho[i0 - 1, p.floor_t:p.floor_t + p.trench_d] = 3e6
    res = dict(params=asdict(p), solid=solid, mask=mask, rho_raw=rho, t_conv=1e-3, stopped=False, circuit=circuit)
    before = rho.copy()
    d = probe_vertical_ions(res, log=None, device=cuda_device)
    assert d["rf_cycle"]
    np.testing.assert_array_equal(d["charged"]["launch_phase"], d["uncharged"]["launch_phase"])
    assert np.max(np.abs(d["charged"]["final_phase"] - d["charged"]["launch_phase"])) > 1
    np.testing.assert_array_equal(res["rho_raw"], before)
    for label in ("charged", "uncharged"):
        assert d[label]["hits"].sum() + d[label]["escaped"] + d[label]["lost"] == p.probe_ions


def test_tapered_monitors_partition_the_walls_and_catch_every_vertical_ion(cuda_device):
    """tests/test_taper.py:92-110: on a tapered trench the monitors include the horizontal steps,
    the height bands partition each sidewall, and every ion of an uncharged vertical beam lands
    on a sidewall, the floor or the mask (40 / 40 / 48 of 224 on the sidewalls and floor)."""
    from trench_b200 import steady
    from trench_b200.probe import probe_vertical_ions
    tr, ma = np.degrees(np.arctan(0.25)), np.degrees(np.arctan(0.5))
    p = replace(Params(), nx=40, trench_w=16, trench_d=20, floor_t=4, mask_t=12, n_vac=10, trench_taper_deg=tr,
                mask_taper_deg=ma, bias="dc", sigma_s=0, n_batches=3, n_per_batch=256, max_steps=800,
                probe_ions=224, probe_trajectories=12)
    solid, mask, i0, i1 = geometry.build_geometry(p)
    regions = steady.charge_monitors(solid, mask, i0, i1, p)
    left = np.unravel_index(regions["left"], solid.shape)
    assert len(np.unique(left[0])) > 1
    res = dict(params=asdict(p), solid=solid, mask=mask, rho_raw=np.zeros(solid.shape), t_conv=1e-3, stopped=False)
    hits = probe_vertical_ions(res, log=None, device=cuda_device)["uncharged"]["hits"]
    flat = hits.ravel()
    assert flat[regions["left"]].sum() + flat[regions["right"]].sum() + flat[regions["bottom"]].sum() \
        + hits[mask].sum() == p.probe_ions
    for side in ("left", "right"):
        bands = [regions[f"{side} band {b}"] for b in (1, 2, 3)]
        np.testing.assert_array_equal(np.sort(np.concatenate(bands)), regions[side])
    assert (flat[regions["left"]].sum(), flat[regions["right"]].sum(), flat[regions["bottom"]].sum()) == (40, 40, 48)
