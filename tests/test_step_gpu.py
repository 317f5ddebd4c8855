"""Multigrid solver and device batch loop against the reference (golden fixtures) and the oracle.

Mirrors the reference's own checks: Poisson solutions (tests/test_features.py:39-49,
65-76), leakage conservation (tests/test_taper.py:112-130) and whole-run CPU/CUDA
agreement (tests/test_cuda.py:106-119).
"""
from dataclasses import replace

import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle_fields as OF
from oracle import oracle_trace as OT
from trench_b200 import geometry, inject
from trench_b200.step import CLAIM_ORDERS
from trench_b200.params import EPS0, Params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case_cls(cuda_device):
    from trench_b200.step import ChargingCase
    return ChargingCase


@pytest.mark.parametrize("name", ["floating", "fixed", "dielectric", "cfg2"])
def test_solver_matches_reference_lu(case_cls, name):
    """Potential of a given charge: multigrid vs the reference's LU within 1e-9 V
    (the accuracy bar is 1e-3 V); leakage operator and conductor response likewise."""
    g = load_golden(f"fields_{name}.npz")
    p = g["p"]
    case = case_cls(replace(p, n_batches=1), green="f64")
    np.testing.assert_allclose(case.external, g["external"], rtol=0, atol=1e-9)
    phi = case.solver.solve((-g["rho"] / EPS0).ravel()).reshape(g["rho"].shape) + case.external
    np.testing.assert_allclose(phi, g["phi"], rtol=0, atol=1e-9)
    np.testing.assert_array_equal(case.S, g["leak_flat"])
    M = case.leak_M.cpu().numpy()
    if "leak_M" in g:
        np.testing.assert_allclose(M, g["leak_M"], rtol=0, atol=1e-10)
    else:
        q = np.random.default_rng(11).normal(size=(case.m, 4))
        np.testing.assert_allclose(M @ q, g["leak_MQ"], rtol=1e-10, atol=1e-10)
    # leakage conserves charge (tests/test_taper.py:119-125)
    np.testing.assert_allclose(M.sum(axis=0), 1.0, rtol=0, atol=1e-9)
    if "g_cond" in g:
        np.testing.assert_allclose(case.g_cond, g["g_cond"], rtol=1e-9, atol=0)
        assert case.C_cond == pytest.approx(float(g["C_cond"]), rel=1e-9)


@pytest.mark.parametrize("shape", ["large_dielectric", "medium_floating"])
def test_solver_matches_reference_lu_on_large_grids(cuda_device, shape):
    """The 400x1400 fine-grid geometry (560,000 cells, dielectric mask) and a 200x700
    floating conductive mask: multigrid (residual target 5e-16 sqrt(n)) against the
    oracle's sparse LU (the reference's solver) for the external potential and a random
    surface charge of tens of volts, within 1e-6 V."""
    from trench_b200.fields import setup_fields
    if shape == "large_dielectric":
        p = replace(Params(), dx=1.25e-9, nx=400, trench_w=40, trench_d=800, floor_t=20, mask_t=80, n_vac=500,
                    mask_type="dielectric", bias="dc", field_mode="floating")
    else:
        p = replace(Params(), dx=2.5e-9, nx=200, trench_w=40, trench_d=400, floor_t=20, mask_t=80, n_vac=200,
                    mask_type="conductor", bias="dc", field_mode="floating")
    solid, mask, _, _ = geometry.build_geometry(p)
    want = OF.setup_fields(p, solid, mask)
    got = setup_fields(p, solid, mask, device=cuda_device)
    np.testing.assert_allclose(got["external"], want["external"], rtol=0, atol=1e-6)
    rho = np.where(OF.surface_cells(solid), np.random.default_rng(2).normal(size=solid.shape), 0.0) * 1e7
    b = (-rho / EPS0).ravel()
    ref = want["solve"](b)
    assert np.abs(ref).max() > 1.0
    np.testing.assert_allclose(got["solve"](b), ref, rtol=0, atol=1e-6)


@pytest.mark.parametrize("name", ["floating", "dielectric", "cfg2"])
def test_green_operator_reproduces_solve(case_cls, name):
    """phi = external + G rho_s on every row cell, for an arbitrary surface charge."""
    g = load_golden(f"fields_{name}.npz")
    p = g["p"]
    for green, tol in (("f64", 1e-9), ("f32", 1e-4)):
        case = case_cls(replace(p, n_batches=1), green=green)
        import torch
        case.rho_s.copy_(torch.from_numpy(g["rho"].ravel()[case.S]))
        case._potential()
        got = case.phi.cpu().numpy()[case.rows]
        np.testing.assert_allclose(got, g["phi"].ravel()[case.rows], rtol=0, atol=tol)
        ex, ey = case.fields()
        if green == "f64":
            np.testing.assert_allclose(ex, g["Ex"], rtol=1e-9, atol=1.0)
            np.testing.assert_allclose(ey, g["Ey"], rtol=1e-9, atol=1.0)
        else:
            # FP32 storage of G: the field carries FP32 noise, bounded relative to the field scale
            scale = max(np.abs(g["Ex"]).max(), np.abs(g["Ey"]).max())
            assert np.abs(ex - g["Ex"]).max() <= 1e-4 * scale
            assert np.abs(ey - g["Ey"]).max() <= 1e-4 * scale


def test_solver_linear_profile_in_homogeneous_medium(case_cls):
    """trench tests/test_features.py:39-49: Dirichlet potentials give a linear profile."""
    from trench_b200.fields import FieldSolver
    from trench_b200.tracer import Context
    p = replace(Params(), nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, bias="dc",
                field_mode="fixed", substrate_voltage=-12, top_voltage=8)
    solid = np.zeros((p.nx, 25), dtype=bool)
    ctx = Context(~solid, 0, p.dx)
    s = FieldSolver(ctx, p, np.ones(solid.shape), np.zeros_like(solid), True)
    from trench_b200.fields import boundary_rhs
    ext = s.solve(boundary_rhs(p, np.ones(solid.shape), dict(substrate=-12, top=8, mask=0)).ravel())
    y = (np.arange(25) + 0.5) / 25
    np.testing.assert_allclose(ext.reshape(solid.shape), np.broadcast_to(-12 + 20 * y, solid.shape), atol=1e-10)


@pytest.mark.parametrize("name", ["floating_leak", "floating_noleak", "fixed_leak", "dielectric_leak",
                                  "absorb_leak", "taper_leak"])
def test_fp64_batch_loop_matches_reference_run(case_cls, name):
    """FP64 tracer + FP64 Green's operator: the reference run() to 1e-10 relative
    (the reference's own CPU/CUDA bar, tests/test_cuda.py:114-119)."""
    g = load_golden(f"run_{name}.npz")
    p = g["p"]
    case = case_cls(p, precision="f64", green="f64")
    res = case.run()
    np.testing.assert_allclose(res["rho_raw"], g["rho_raw"], rtol=1e-10, atol=1e-8)
    np.testing.assert_allclose(res["mean_phi"], g["mean_phi"], rtol=1e-10, atol=1e-8)
    for k in ("ratio_i_bottom", "ratio_e_bottom", "esc_e", "lost"):
        np.testing.assert_array_equal(res["hist"][k], g[f"hist_{k}"])
    np.testing.assert_allclose(res["hist"]["leak"], g["hist_leak"], rtol=1e-9, atol=1e-12)
    for k in case.probes:
        np.testing.assert_allclose(res["hist"][k], g[f"hist_{k}"], rtol=1e-10, atol=1e-8)
    check_display(res, g)


def check_display(res, g):
    """The result's display outputs: potential, charge with the conductor's induced
    surface charge (trench_charging_2d.py:833-843), external potential, field, voltages."""
    np.testing.assert_allclose(res["phi"], g["phi_display"], rtol=1e-10, atol=1e-8)
    np.testing.assert_allclose(res["external_phi"], g["external_phi"], rtol=1e-10, atol=1e-8)
    scale = np.abs(g["rho_display"]).max()
    np.testing.assert_allclose(res["rho"], g["rho_display"], rtol=1e-8, atol=1e-9 * scale)
    escale = max(np.abs(g["Ex_display"]).max(), np.abs(g["Ey_display"]).max())
    np.testing.assert_allclose(res["Ex"], g["Ex_display"], rtol=1e-8, atol=1e-9 * escale)
    np.testing.assert_allclose(res["Ey"], g["Ey_display"], rtol=1e-8, atol=1e-9 * escale)
    np.testing.assert_allclose([res["voltages"][k] for k in ("substrate", "mask", "top")], g["volts"],
                               rtol=1e-12, atol=1e-12)


def test_fp32_batch_loop_tracks_oracle(case_cls):
    """FP32 tracer + FP64 Green's operator over 5 batches of the AR-8 geometry with
    2^14 particles per species: bottom ion flux within 3 sigma of the FP64 oracle
    batch loop fed the same injected particles, potentials within 1% of the swing."""
    p = replace(Params(), nx=60, trench_w=20, trench_d=160, floor_t=10, mask_t=20, n_vac=60, trench_taper_deg=2.0,
                mask_taper_deg=5.0, mask_type="dielectric", mask_eps_r=3.0, electron_temp_eV=3.0, bias="dc",
                ion_energy_eV=90.0, n_per_batch=1 << 14, n_batches=5, seed=3)
    case = case_cls(p, precision="f32", green="f64")
    res = case.run()
    solid, mask, _, _ = geometry.build_geometry(p)
    st = OF.BatchState(p, solid, mask)
    rng = np.random.default_rng(p.seed)
    for _ in range(p.n_batches):
        parts = inject.inject(p, p.n_per_batch, solid.shape[1], rng)
        st.step(*OT.trace(*parts, st.Ex, st.Ey, ~solid, p, st.barrier()))
    ri, ro = res["hist"]["ratio_i_bottom"], np.array(st.hist["ratio_i_bottom"])
    norm = p.n_per_batch * (case.b1 - case.b0) / p.nx
    sigma = np.sqrt(np.maximum(ro * norm, 1)) / norm
    assert np.all(np.abs(ri - ro) <= 3 * sigma + 1e-12), (ri, ro)
    swing = np.ptp(st.phi)
    assert np.max(np.abs(res["mean_phi"] - st.phi)) <= 0.01 * swing


def _cfg1_sampler(p):
    return inject.energy_angle_sampler(p, lambda r, k: np.full(k, 100.0), inject.gaussian_angle(2.0))


def test_fp64_batch_loop_matches_reference_cfg1_full_run(case_cls):
    """80x200 floating conductive mask, DC 100 eV ions at N(0, 2 deg), 10k + 10k per
    batch, 30 batches: FP64 tracer + FP64 Green's operator reproduce the reference
    run() (1e-10 relative on charge and potential, exact counts).  The absolute floor
    scales with the largest charge (1.9e7 C/m^3): leakage spreads tails down to 1e-8."""
    g = load_golden("run_cfg1_30.npz")
    p = g["p"]
    case = case_cls(p, precision="f64", green="f64")
    res = case.run(ion_velocity=_cfg1_sampler(p))
    np.testing.assert_allclose(res["rho_raw"], g["rho_raw"], rtol=1e-10, atol=1e-13 * np.abs(g["rho_raw"]).max())
    np.testing.assert_allclose(res["mean_phi"], g["mean_phi"], rtol=1e-10, atol=1e-8)
    for k in ("ratio_i_bottom", "ratio_e_bottom", "esc_e", "lost"):
        np.testing.assert_array_equal(res["hist"][k], g[f"hist_{k}"])
    np.testing.assert_allclose(res["hist"]["leak"], g["hist_leak"], rtol=1e-9, atol=1e-12)


def test_fp32_batch_loop_tracks_reference_cfg1_full_run(case_cls):
    """Same 30-batch run with the FP32 tracer: per-batch bottom ion flux within
    3 sigma of the reference (counting noise of the batch), the final surface
    charge's total within 1%, and the final potential within 2% of its swing on
    every cell.  After the first hit that differs from the FP64 run the two runs
    are different Monte Carlo samples of the same charging, so their potentials
    differ by the charging noise; the 1e-3 V bar holds for one batch from a common
    charge (test_accuracy_gpu.py)."""
    g = load_golden("run_cfg1_30.npz")
    p = g["p"]
    case = case_cls(p, precision="f32", green="f64")
    res = case.run(ion_velocity=_cfg1_sampler(p))
    ri, ro = res["hist"]["ratio_i_bottom"], g["hist_ratio_i_bottom"]
    norm = p.n_per_batch * (case.b1 - case.b0) / p.nx
    sigma = np.sqrt(np.maximum(ro * norm, 1)) / norm
    assert np.all(np.abs(ri - ro) <= 3 * sigma + 1e-12), (ri, ro)
    tot_ref, tot = g["rho_raw"].sum(), res["rho_raw"].sum()
    assert abs(tot - tot_ref) <= 0.01 * abs(g["rho_raw"]).sum()
    swing = np.ptp(g["mean_phi"])
    assert np.max(np.abs(res["mean_phi"] - g["mean_phi"])) <= 0.02 * swing


@pytest.mark.parametrize("name", ["floating", "dielectric"])
def test_until_steady_stops_where_the_reference_does(case_cls, name):
    """run() with until_steady (FP64 tracer): the steady-state check passes at the same
    batch as the reference run(), with the
    same potential and charge-monitor histories and the same steady values."""
    g = load_golden(f"steady_run_{name}.npz")
    p = g["p"]
    case = case_cls(p, precision="f64", green="f64")
    res = case.run()
    assert res["converged"] == bool(g["converged"])
    assert res["t_conv"] == pytest.approx(float(g["t_conv"]), rel=1e-12)
    assert len(res["hist"]["t"]) == len(g["hist_t"])
    for k in ("ratio_i_bottom", "ratio_e_bottom", "esc_e", "lost"):
        np.testing.assert_array_equal(res["hist"][k], g[f"hist_{k}"])
    for k in case.probes:
        np.testing.assert_allclose(res["hist"][k], g[f"hist_{k}"], rtol=1e-10, atol=1e-8)
    for k, v in res["charge_monitor_hist"].items():
        want = g[f"monitor_{k}"]
        np.testing.assert_allclose(v, want, rtol=1e-9, atol=1e-9 * max(np.abs(want).max(), 1e-30))
    for k in ("left", "right"):
        np.testing.assert_allclose(res["charge_hist"][k], g[f"charge_{k}"], rtol=1e-9, atol=1e-25)
    want = dict(zip([str(n) for n in g["steady_names"]], g["steady_values"]))
    for k, v in res["steady"].items():
        assert v == pytest.approx(want[k], rel=1e-10, abs=1e-8)
    assert res["checkpoint"]["steady_n_ok"] == int(g["steady_n_ok"])
    np.testing.assert_allclose(res["rho_raw"], g["rho_raw"], rtol=1e-10, atol=1e-13 * np.abs(g["rho_raw"]).max())


def test_device_injected_run_replays_like_eager_batches(case_cls):
    """run(injector=...) (inject + step replayed from one CUDA graph) equals the same
    batches injected and stepped one by one."""
    import torch
    from trench_b200 import inject as inj_mod
    p = replace(Params(), nx=30, trench_w=10, trench_d=20, floor_t=5, mask_t=6, n_vac=12, bias="dc",
                sigma_s=1e-14, n_per_batch=3000, n_batches=6)
    et = inj_mod.table_from_pdf(inj_mod.bimodal_gaussian_pdf(40.0, 6.0, 140.0, 6.0), 0.0, 200.0, bins=64)
    a, b = case_cls(p), case_cls(p)
    ia = inj_mod.DeviceInjector(a, seed=5, energy_table=et)
    ib = inj_mod.DeviceInjector(b, seed=5, energy_table=et)
    res = a.run(injector=ia)
    for _ in range(p.n_batches):
        ib()
        b.step()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(res["rho_raw"], b.rho())
    hb = b.history()
    for k in res["hist"]:
        np.testing.assert_array_equal(res["hist"][k], hb[k])
    np.testing.assert_array_equal(res["charge_monitor_hist"]["left"], b.charge_history()["left"])


def test_graph_replay_equals_eager(case_cls):
    """A captured batch replays the same kernels: same counts as an eager batch."""
    import torch
    p = replace(Params(), nx=30, trench_w=10, trench_d=20, floor_t=5, mask_t=6, n_vac=12, bias="dc",
                sigma_s=1e-14, n_per_batch=2000, n_batches=4)
    a = case_cls(p, precision="f32")
    b = case_cls(p, precision="f32")
    parts = inject.inject(p, p.n_per_batch, a.ny, np.random.default_rng(9))
    a.load(*parts)
    b.load(*parts)
    a.step()
    b.capture()
    torch.cuda.synchronize()
    # capture ran nothing; replays do the work
    for _ in range(2):
        a.load(*parts)
        a.step()
    b.replay()
    b.replay()
    b.replay()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a.rho(), b.rho())
    np.testing.assert_array_equal(a.history()["ratio_i_bottom"], b.history()["ratio_i_bottom"])


def test_rf_batch_loop_matches_reference_run(case_cls):
    """circuit_rf on the device: basis fields, launch phases and the in-flight clock
    (FP64 kernel) reproduce the reference run() (tests/test_taper.py:273-294)."""
    g = load_golden("run_rf_taper.npz")
    p = g["p"]
    circuit = dict(t=g["circuit_t"], uw=g["circuit_uw"], um=g["circuit_um"], up=g["circuit_up"], V1=g["circuit_V1"])
    case = case_cls(p, precision="f64", green="f64", circuit=circuit)
    res = case.run()
    np.testing.assert_allclose(res["rho_raw"], g["rho_raw"], rtol=1e-10, atol=1e-6)
    np.testing.assert_allclose(res["mean_phi"], g["mean_phi"], rtol=1e-10, atol=1e-8)
    for k in ("ratio_i_bottom", "ratio_e_bottom", "esc_e", "lost"):
        np.testing.assert_array_equal(res["hist"][k], g[f"hist_{k}"])
    check_display(res, g)


def test_rf_batch_loop_in_fp32(case_cls):
    """circuit_rf with the FP32 tracer (in-flight clock in FP32): the same run as the
    reference's within the FP32 tracer's per-particle disagreement: the deposited charge
    differs by at most 1% (L1) and the bottom ion ratio of each batch by at most 2 ions."""
    g = load_golden("run_rf_taper.npz")
    p = g["p"]
    circuit = dict(t=g["circuit_t"], uw=g["circuit_uw"], um=g["circuit_um"], up=g["circuit_up"], V1=g["circuit_V1"])
    case = case_cls(p, precision="f32", green="f64", circuit=circuit)
    res = case.run()
    d = np.abs(res["rho_raw"] - g["rho_raw"]).sum() / np.abs(g["rho_raw"]).sum()
    print(f"FP32 RF run: L1 charge difference {d:.2e}")
    assert d <= 0.01, d
    np.testing.assert_allclose(res["hist"]["ratio_i_bottom"], g["hist_ratio_i_bottom"], atol=2.0 / p.n_per_batch)


@pytest.mark.parametrize("mode", ["floating", "fixed", "dielectric"])
def test_resume_equals_continuous_run(case_cls, tmp_path, mode):
    """Split-and-resume equals the continuous run bit for bit (tests/test_resume.py:35-49),
    through the NPZ file."""
    p = replace(Params(), nx=30, trench_w=10, trench_d=20, floor_t=5, mask_t=6, n_vac=12, bias="dc",
                sigma_s=1e-14, n_per_batch=1500, n_batches=3, seed=4)
    if mode == "fixed":
        p = replace(p, field_mode="fixed", substrate_voltage=-20, mask_voltage=-10)
    elif mode == "dielectric":
        p = replace(p, mask_type="dielectric")
    full = case_cls(p, max_batches=4).run()
    a = case_cls(p, max_batches=4)
    rng = np.random.default_rng(p.seed)
    a.run(n_batches=1, rng=rng)
    a.save(tmp_path / "part.npz", rng=rng)
    b = case_cls(p, max_batches=4)
    cont = b.run(n_batches=2, resume=case_cls.load_checkpoint(tmp_path / "part.npz"))
    np.testing.assert_array_equal(cont["rho_raw"], full["rho_raw"])
    np.testing.assert_array_equal(cont["mean_phi"], full["mean_phi"])
    np.testing.assert_array_equal(cont["Ex"], full["Ex"])
    for k in full["hist"]:
        np.testing.assert_array_equal(cont["hist"][k], full["hist"][k])


def test_resume_from_a_reference_result(case_cls):
    """A reference run() result (rho_raw, history, PCG64 state) continues on the device:
    the state after 4 reference batches, restored, gives the reference's next potentials."""
    g = load_golden("run_floating_leak.npz")
    p = g["p"]
    case = case_cls(p, precision="f64", max_batches=8)
    hist = {k[5:]: g[k] for k in g if k.startswith("hist_")}
    case.restore(dict(rho_raw=g["rho_raw"], hist=hist))
    np.testing.assert_allclose(case.full_potential(), g["mean_phi"], rtol=1e-10, atol=1e-8)
    assert case.batches_done() == p.n_batches


def test_host_pipeline_equals_sequential_batches(case_cls):
    """Copies overlapped with compute (two buffer sets, one graph each) give the same
    results as loading and stepping one batch after the other."""
    import torch
    from trench_b200.step import HostPipeline
    p = replace(Params(), nx=30, trench_w=10, trench_d=20, floor_t=5, mask_t=6, n_vac=12, bias="dc",
                sigma_s=1e-14, n_per_batch=3000, n_batches=4)
    rng = np.random.default_rng(8)
    a, b = case_cls(p, max_batches=6), case_cls(p, max_batches=6)
    host = [[torch.from_numpy(np.ascontiguousarray(v)).pin_memory()
             for v in inject.inject(p, p.n_per_batch, a.ny, rng)] for _ in range(4)]
    for h in host:
        a.load(*h)
        a.step()
    b.load(*host[0])
    rows = torch.empty((4, b.hist_cols), dtype=torch.float64).pin_memory()
    HostPipeline(b, 2 * p.n_per_batch).run(host, rows)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a.rho(), b.rho())
    np.testing.assert_array_equal(rows.numpy(), b.hist[:4].cpu().numpy())
    np.testing.assert_array_equal(a.history()["ratio_e_bottom"], b.history()["ratio_e_bottom"])
    # batches without qm (the species' ratios written on the device) give the same run
    c = case_cls(p, max_batches=6)
    c.load(*host[0])
    rows_c = torch.empty((4, c.hist_cols), dtype=torch.float64).pin_memory()
    HostPipeline(c, 2 * p.n_per_batch).run([h[:4] + h[5:] for h in host], rows_c)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(c.rho(), b.rho())
    np.testing.assert_array_equal(rows_c.numpy(), rows.numpy())
    with pytest.raises(ValueError):
        HostPipeline(c, 2 * p.n_per_batch).run([h[:3] for h in host])


def test_autotuners_pick_a_shape_and_keep_results(case_cls):
    """Every tracer launch shape gives the same counts (deterministic tracing); the
    multigrid schedule autotuner keeps the solution."""
    import torch
    p = replace(Params(), nx=60, trench_w=20, trench_d=80, floor_t=10, mask_t=20, n_vac=40, bias="dc",
                mask_type="dielectric", n_per_batch=20000, n_batches=2)
    tuned = case_cls(p, autotune=True)
    plain = case_cls(p)
    np.testing.assert_allclose(tuned.external, plain.external, rtol=0, atol=1e-9)
    parts = inject.inject(p, p.n_per_batch, tuned.ny, np.random.default_rng(3))
    tuned.load(*parts)
    timings = tuned.autotune_tracer()
    assert set(timings) == {(t, c, o) for t, c in tuned.TRACER_SHAPES for o in range(len(CLAIM_ORDERS))}
    counts, hits = [], []
    from trench_b200 import _capi
    tuned.hit = torch.full((tuned.capacity,), -1, dtype=torch.int32, device=tuned.dev)
    for t, c, o in sorted(timings):
        assert _capi.lib().tb_set_tuning(tuned.ctx.handle, t, c) == 0
        assert _capi.lib().tb_set_claim_order(tuned.ctx.handle, o) == 0
        tuned._trace_only(2 * p.n_per_batch)
        torch.cuda.synchronize()
        counts.append(tuned.counts.cpu().numpy().copy())
        hits.append(torch.where(tuned.status[:2 * p.n_per_batch] == 1, tuned.hit[:2 * p.n_per_batch], -1).cpu().numpy())
    for c, h in zip(counts[1:], hits[1:]):
        np.testing.assert_array_equal(c, counts[0])
        np.testing.assert_array_equal(h, hits[0])
    assert "poisson_schedule" in tuned.tuning and "tracer_shape" in tuned.tuning
    assert tuned.tuning["claim_order"] in CLAIM_ORDERS
    assert _capi.lib().tb_set_claim_order(tuned.ctx.handle, len(CLAIM_ORDERS)) == _capi.TB_ERR_ARG


class _StopAfter:
    """A stop flag that is raised after `k` checks (the loop checks it before each batch)."""

    def __init__(self, k):
        self.k = k

    def is_set(self):
        self.k -= 1
        return self.k < 0


def test_stop_during_resume_keeps_the_last_batch_and_can_resume_again(case_cls):
    """tests/test_resume.py:196-206: a resumed run stopped between batches returns a result that
    resumes again, and the pieces together equal the continuous run bit for bit."""
    p = replace(Params(), nx=30, trench_w=10, trench_d=20, floor_t=5, mask_t=6, n_vac=12, bias="dc",
                sigma_s=1e-14, n_per_batch=800, n_batches=3, seed=6)
    full = case_cls(replace(p, n_batches=8), max_batches=10).run()
    part = case_cls(p, max_batches=10).run()
    interrupted = case_cls(p, max_batches=10).run(resume=part, stop=_StopAfter(1))
    assert interrupted["stopped"] and len(interrupted["hist"]["t"]) == 4
    resumed = case_cls(replace(p, n_batches=4), max_batches=10).run(resume=interrupted)
    np.testing.assert_array_equal(resumed["rho_raw"], full["rho_raw"])
    for k in full["hist"]:
        np.testing.assert_array_equal(resumed["hist"][k], full["hist"][k])
