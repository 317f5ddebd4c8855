"""Boundary conditions and driven electrodes of the device field solve and batch loop,
restated from the reference's tests/test_features.py:51-200 on this backend."""
from dataclasses import asdict, replace

import numpy as np
import pytest

from trench_b200 import geometry
from trench_b200.params import AMU, E_CHARGE, Params

pytestmark = pytest.mark.gpu


def small_params(**changes):
    base = dict(nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, bias="dc", sigma_s=0, n_batches=3,
                n_per_batch=200, max_steps=800, probe_ions=120, probe_trajectories=8)
    return replace(Params(), **{**base, **changes})


def fake_circuit():
    return dict(t=np.arange(4) * 1e-8, uw=np.array([-80.0, -100.0, -80.0, -60.0]),
                um=np.array([-40.0, -50.0, -40.0, -30.0]), up=np.full(4, 10.0), V1=np.array([50.0, 60.0, 50.0, 40.0]))


def test_fixed_mask_stays_fixed_with_charge_and_leakage(cuda_device):
    from trench_b200.step import ChargingCase
    p = small_params(field_mode="fixed", substrate_voltage=-30, mask_voltage=-10, sigma_s=1e-14)
    res = ChargingCase(p, device=cuda_device).run()
    mask = res["mask"]
    np.testing.assert_allclose(res["phi"][mask], -10, atol=1e-10)
    assert np.all(res["rho_raw"][mask] == 0)
    assert np.any(np.abs(res["rho"][mask]) > 0)        # the induced charge is shown
    assert np.any(np.abs(res["rho_raw"][~mask]) > 0)
    _, _, i0, i1 = geometry.build_geometry(p)
    for side, ix in (("left", i0 - 1), ("right", i1)):
        assert len(res["charge_hist"][side]) == p.n_batches
        np.testing.assert_allclose(res["charge_hist"][side][-1],
                                   res["rho_raw"][ix, p.floor_t:p.floor_t + p.trench_d].sum() * p.dx ** 2)


def test_pillar_boundary_reproduces_linear_dielectric_voltage(cuda_device):
    """A SiO2 slab under an equipotential electrode: the pillar sides carry the same linear
    potential as the slab's interior."""
    from trench_b200.fields import setup_fields
    p = small_params(field_mode="fixed", side_bc="pillar", substrate_voltage=-20, mask_voltage=10)
    ny = p.floor_t + p.trench_d + p.mask_t + p.n_vac
    solid = np.zeros((p.nx, ny), dtype=bool)
    top = p.floor_t + p.trench_d
    solid[:, :top + p.mask_t] = True
    mask = np.zeros_like(solid)
    mask[:, top:top + p.mask_t] = True
    f = setup_fields(p, solid, mask, device=cuda_device)
    expected = -20 + 30 * (np.arange(top) + 0.5) / top
    np.testing.assert_allclose(f["external"][:, :top], np.broadcast_to(expected, (p.nx, top)), atol=1e-10)


def test_left_and_right_fixed_boundaries_are_distinct(cuda_device):
    from trench_b200.fields import setup_fields
    p = small_params(field_mode="fixed", side_bc="fixed", left_voltage=20, right_voltage=-20)
    solid, mask, _, _ = geometry.build_geometry(p)
    f = setup_fields(p, solid, mask, device=cuda_device)
    ext = f["external"]
    assert ext[0, 8] > 0 and ext[-1, 8] < 0
    np.testing.assert_allclose(ext, -ext[::-1], atol=1e-10)
    ce = f["solver"].ce
    assert ce[-1, 8] == 0            # the SiO2 ends have no periodic coupling
    assert ce[-1, -1] != 0           # the vacuum on top stays periodic


def test_circuit_mode_applies_phase_and_avoids_double_acceleration(cuda_device):
    """The frozen circuit field at rf_phase 90: mask at -60 V, substrate -110 V, and ions enter at
    the Bohm energy Te/2 rather than with the sheath's IED."""
    from trench_b200.step import ChargingCase
    p = small_params(field_mode="circuit", side_bc="pillar", rf_phase=90, bias="rf")
    case = ChargingCase(p, device=cuda_device, circuit=fake_circuit())
    res = case.run()
    np.testing.assert_allclose(res["phi"][res["mask"]], -60)
    assert res["voltages"]["substrate"] == -110
    # the last batch's ions as injected (a particle stopped at the step cap has its state written back)
    injected = case.status[:p.n_per_batch].cpu().numpy() != 3
    vy = case.X[3][:p.n_per_batch].cpu().numpy()[injected]
    assert injected.sum() > p.n_per_batch // 2
    energy = 0.5 * p.ion_mass_amu * AMU * vy ** 2 / E_CHARGE
    np.testing.assert_allclose(energy, p.electron_temp_eV / 2, rtol=1e-12)


def test_probe_phase_changes_the_field_but_not_the_stored_charge(cuda_device):
    from trench_b200.probe import probe_vertical_ions
    p = small_params(field_mode="circuit", side_bc="pillar", bias="rf")
    solid, mask, _, _ = geometry.build_geometry(p)
    res = dict(params=asdict(p), solid=solid, mask=mask, rho_raw=np.zeros(solid.shape), t_conv=1e-3, stopped=False,
               circuit=fake_circuit())
    original = res["rho_raw"].copy()
    probe = probe_vertical_ions(res, phase=90, log=None, device=cuda_device)
    assert probe["phase"] == 90
    np.testing.assert_allclose(probe["charged"]["phi"][mask], -60)
    np.testing.assert_array_equal(res["rho_raw"], original)
    assert res["params"]["rf_phase"] == 0


def test_driven_leakage_responds_to_voltage_without_particle_charge(cuda_device):
    from trench_b200.step import ChargingCase
    p = small_params(field_mode="fixed", side_bc="pillar", substrate_voltage=-20, mask_voltage=-10, flux=1e-10,
                     n_batches=1, sigma_s=1e-14)
    res = ChargingCase(p, device=cuda_device).run()
    assert np.max(np.abs(res["rho_raw"])) > 1e6     # surface current driven by the electrode voltages
    np.testing.assert_allclose(res["phi"][res["mask"]], -10)
