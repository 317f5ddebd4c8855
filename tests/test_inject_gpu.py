"""Device-side injection: the Philox stream equals the host restatement, and the
sampled distributions are those of the reference's inject (trench_charging_2d.py:458-489)."""
import ctypes
from dataclasses import replace

import numpy as np
import pytest

from trench_b200 import inject
from trench_b200.params import AMU, E_CHARGE, M_E, Params

pytestmark = pytest.mark.gpu


def small_case(n, cuda_device):
    from trench_b200.step import ChargingCase
    p = replace(Params(), nx=30, trench_w=10, trench_d=20, floor_t=5, mask_t=6, n_vac=12, bias="dc", sigma_s=0,
                n_per_batch=n, electron_temp_eV=3.0, ion_energy_eV=90.0)
    return ChargingCase(p, device=cuda_device)


def test_device_philox_equals_host(cuda_device):
    import torch
    from trench_b200 import _capi
    case = small_case(16, cuda_device)
    n, seed, batch = 4096, 0x0123456789ABCDEF, 77
    out = torch.zeros(4 * n, dtype=torch.int32, device=case.dev)
    code = _capi.lib().tb_philox_fill(case.ctx.handle, seed, batch, n, ctypes.c_void_p(out.data_ptr()), None)
    assert code == 0
    got = out.cpu().numpy().view(np.uint32).reshape(n, 4)
    ctr = np.stack([np.arange(n), np.full(n, batch & 0xffffffff), np.full(n, batch >> 32), np.zeros(n)], axis=1)
    want = inject.philox4x32_10(ctr.astype(np.uint64), (seed & 0xffffffff, seed >> 32))
    np.testing.assert_array_equal(got, want)


def test_device_injection_distributions(cuda_device):
    n = 1 << 18
    case = small_case(n, cuda_device)
    p = case.p
    et = inject.table_from_pdf(inject.bimodal_gaussian_pdf(40, 6, 140, 6), 0, 200)
    at = inject.table_from_pdf(inject.half_gaussian_pdf(np.radians(3.0)), 0, np.radians(15.0))
    inj = inject.DeviceInjector(case, seed=5, energy_table=et, angle_table=at)
    inj(0)
    x, y, vx, vy, qm = (t[:2 * n].cpu().numpy() for t in case.X)
    spc = case.SPC[:2 * n].cpu().numpy()
    assert (spc[:n] == 0).all() and (spc[n:] == 1).all()
    lx, ly = p.nx * p.dx, case.ny * p.dx
    assert (x >= 0).all() and (x < lx).all() and np.all(y == ly - 1e-3 * p.dx)
    assert abs(x.mean() / lx - 0.5) < 0.01
    m_i = p.ion_mass_amu * AMU
    np.testing.assert_allclose(qm[:n], E_CHARGE / m_i)
    np.testing.assert_allclose(qm[n:], -E_CHARGE / M_E)
    # ions: energy follows the table, angles are a symmetric half-Gaussian pair
    e = 0.5 * m_i * (vx[:n] ** 2 + vy[:n] ** 2) / E_CHARGE
    hist, _ = np.histogram(e, bins=et[0][::16])
    want = np.diff(et[1][::16]) * n
    ok = want > 50
    assert np.all(np.abs(hist[ok] - want[ok]) < 5 * np.sqrt(want[ok]) + 5)
    th = np.degrees(np.arctan2(vx[:n], -vy[:n]))
    assert abs(th.mean()) < 0.05 and abs(np.abs(th).mean() - 3.0 * np.sqrt(2 / np.pi)) < 0.05
    # electrons: flux-weighted Maxwellian (normal tangential, Rayleigh normal component)
    s = np.sqrt(p.electron_temp_eV * E_CHARGE / M_E)
    assert abs(vx[n:].mean()) < 0.01 * s and abs(vx[n:].std() / s - 1) < 0.01
    assert abs(-vy[n:].mean() / (s * np.sqrt(np.pi / 2)) - 1) < 0.01
    # a different batch counter gives different particles, the same one the same
    first = x.copy()
    inj(1)
    assert not np.array_equal(case.X[0][:2 * n].cpu().numpy(), first)
    inj(0)
    np.testing.assert_array_equal(case.X[0][:2 * n].cpu().numpy(), first)


def test_device_injection_feeds_the_batch_loop(cuda_device):
    """A batch with device injection runs through the same step (all particles accounted)."""
    case = small_case(4000, cuda_device)
    inj = inject.DeviceInjector(case, seed=3)
    for b in range(3):
        inj(b)
        case.step()
    case.check()
    h = case.history()
    assert len(h["ratio_i_bottom"]) == 3 and np.all(h["particle_steps"] > 0)


def test_device_injection_rf_launch_phases(cuda_device):
    """circuit_rf: the injector writes stratified launch times (each species covers the
    period with one particle per stratum, trench_rf.py:14-18), zero flight time, and ions
    at the Bohm energy Te/2 (trench_charging_2d.py:1135-1139); a run replayed from the
    device injector accounts for every particle."""
    from conftest import load_golden
    from trench_b200.step import ChargingCase
    g = load_golden("run_rf_taper.npz")
    circuit = dict(t=g["circuit_t"], uw=g["circuit_uw"], um=g["circuit_um"], up=g["circuit_up"], V1=g["circuit_V1"])
    p = replace(g["p"], n_per_batch=2000, n_batches=4)
    case = ChargingCase(p, device=cuda_device, circuit=circuit)
    n, period = p.n_per_batch, case.rf["period"]
    inj = inject.DeviceInjector(case, seed=9)
    inj(0)
    clock = case.clock[:2 * n].cpu().numpy()
    assert np.all(clock[:, 1] == 0) and np.all((clock[:, 0] >= 0) & (clock[:, 0] < period))
    for s in (slice(0, n), slice(n, 2 * n)):
        np.testing.assert_array_equal(np.sort(np.floor(clock[s, 0] / period * n)), np.arange(n))
    vx, vy = (t[:n].cpu().numpy() for t in case.X[2:4])
    m_i = p.ion_mass_amu * AMU
    np.testing.assert_allclose(0.5 * m_i * vy ** 2 / E_CHARGE, p.electron_temp_eV / 2, rtol=1e-12)
    assert abs(vx.std() / np.sqrt(p.ion_temp_eV * E_CHARGE / m_i) - 1) < 0.1
    res = case.run(injector=inject.DeviceInjector(case, seed=10))
    h = res["hist"]
    assert len(h["t"]) == p.n_batches and np.all(np.isfinite(res["mean_phi"]))
    assert np.all(h["particle_steps"] > 0)
