"""circuit_rf superposition: the unit-voltage basis built on the device solver, shifted to
any display phase, equals an independent Poisson solve with the electrode voltages of
that phase (the reference's tests/test_rf_cycle.py:33-45, restated on this backend)."""
from dataclasses import replace

import numpy as np
import pytest

from trench_b200 import geometry
from trench_b200.params import Params

pytestmark = pytest.mark.gpu


def waveform(period=4e-10, amplitude=35.0):
    t = np.arange(256) * period / 256
    up = 10 + 2 * np.cos(2 * np.pi * t / period)
    uw = -80 - amplitude * np.sin(2 * np.pi * t / period) + up
    um = -40 - amplitude / 2 * np.sin(2 * np.pi * t / period) + up
    return dict(t=t, uw=uw, um=um, up=up, V1=up - um)


@pytest.mark.parametrize("side_bc", ["periodic", "pillar", "fixed"])
def test_basis_superposition_matches_independent_solve_at_every_phase(cuda_device, side_bc):
    from trench_b200.fields import field_snapshot, setup_fields
    p = replace(Params(), nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, field_mode="circuit_rf",
                bias="rf", side_bc=side_bc, left_voltage=-20, right_voltage=5, rf_freq=2.5e9, sigma_s=0)
    c = waveform()
    solid, mask, _, _ = geometry.build_geometry(p)
    f = setup_fields(p, solid, mask, c, device=cuda_device)
    scale = np.abs(f["external"]).max()
    for phase in (0, 45, 90, 180, 270, 359.9, 405):
        snapshot, _, rhs, volts = field_snapshot(f, f["external"], replace(p, rf_phase=phase))
        direct = setup_fields(replace(p, field_mode="circuit", rf_phase=phase), solid, mask, c, device=cuda_device)
        # both sides are multigrid solves to a 1e-13 relative residual
        np.testing.assert_allclose(snapshot, direct["external"], atol=1e-9 * scale, rtol=0)
        np.testing.assert_allclose(rhs, direct["boundary_rhs"], atol=1e3, rtol=2e-13)
        assert volts["substrate"] == pytest.approx(direct["volts"]["substrate"])
        assert volts["mask"] == pytest.approx(direct["volts"]["mask"])


def small_rf_params(**changes):
    base = replace(Params(), nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, field_mode="circuit_rf",
                   bias="rf", side_bc="pillar", rf_freq=2.5e9, sigma_s=0, n_batches=3, n_per_batch=128,
                   max_steps=1000)
    return replace(base, **changes)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_constant_wave_reduces_to_frozen_field(cuda_device, precision):
    """A waveform without variation traces like the frozen field (tests/test_rf_cycle.py:116-128):
    the FP64 kernel gives the same status for every particle; the FP32 kernel, whose RF
    step rounds the same arithmetic in another order, the same for all but a few."""
    from trench_b200 import inject
    from trench_b200.fields import compute_field, setup_fields
    from trench_b200.tracer import B200Tracer
    p = small_rf_params()
    solid, mask, _, _ = geometry.build_geometry(p)
    f = setup_fields(p, solid, mask, waveform(amplitude=0), device=cuda_device)
    ex, ey = compute_field(f["external"], ~solid, p, 0)
    args = inject.inject(p, p.n_per_batch, solid.shape[1], np.random.default_rng(1))
    rf = {**f["rf"], "initial_time": np.zeros(2 * p.n_per_batch)}
    t = B200Tracer(~solid, cuda_device, precision=precision)
    t(*args, ex, ey, ~solid, p)
    st_frozen = t.last["status"].copy()
    t(*args, ex, ey, ~solid, p, rf=rf)
    same = t.last["status"] == st_frozen
    if precision == "f64":
        assert same.all()
    else:
        assert same.mean() >= 0.99


def test_display_phase_does_not_change_the_charge(cuda_device):
    """The charging uses the whole waveform; rf_phase only moves the displayed potential
    (tests/test_rf_cycle.py:131-145)."""
    from trench_b200.step import ChargingCase
    p = small_rf_params()
    a = ChargingCase(p, device=cuda_device, circuit=waveform()).run()
    b = ChargingCase(replace(p, rf_phase=90), device=cuda_device, circuit=waveform()).run()
    np.testing.assert_array_equal(a["rho_raw"], b["rho_raw"])
    for key in a["hist"]:
        np.testing.assert_array_equal(a["hist"][key], b["hist"][key])
    assert np.max(np.abs(a["phi"] - b["phi"])) > 10
    np.testing.assert_allclose(a["mean_phi"][a["mask"]], -40, atol=1e-9)


def test_rf_resume_equals_continuous_run(cuda_device):
    """circuit_rf split and resumed (particle and launch-phase generator states carried in the
    checkpoint) equals the continuous run bit for bit (tests/test_resume.py:61-89)."""
    from trench_b200.step import ChargingCase
    p = small_rf_params(n_batches=4, n_per_batch=256)
    c = waveform()
    full = ChargingCase(p, device=cuda_device, circuit=c, max_batches=6).run()
    part = ChargingCase(replace(p, n_batches=2), device=cuda_device, circuit=c, max_batches=6).run()
    resumed = ChargingCase(replace(p, n_batches=2), device=cuda_device, circuit=c, max_batches=6).run(resume=part)
    np.testing.assert_array_equal(resumed["rho_raw"], full["rho_raw"])
    for k in full["hist"]:
        np.testing.assert_array_equal(resumed["hist"][k], full["hist"][k])
