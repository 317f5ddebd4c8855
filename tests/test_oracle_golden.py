"""The oracle (C/NumPy restatement) against the reference's golden outputs.

These pin the checker itself: every fixture was produced by the reference code
(tests/golden/make_golden.py).  CPU only.
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle_fields as OF
from oracle import oracle_trace as OT
from trench_b200 import geometry, inject

TRACE_CASES = ["small_barrier", "small_absorb", "taper_barrier", "taper_absorb", "cfg1", "cfg2", "rf_taper"]


def rf_of(g):
    if "rf_period" not in g:
        return None
    return dict(period=float(g["rf_period"]), dt_max=float(g["rf_dt_max"]), wave=g["rf_wave"], phi=g["rf_phi"],
                Ex=g["rf_Ex"], Ey=g["rf_Ey"], initial_time=g["rf_initial_time"])


def trace_args(g):
    bar = (g["phi"], g["wface"]) if bool(g["barrier"]) else None
    return ([g[k].copy() for k in ("x", "y", "vx", "vy", "qm", "spc")], g["Ex"], g["Ey"], ~g["solid"], g["p"], bar)


@pytest.mark.parametrize("name", TRACE_CASES)
def test_oracle_trace_matches_reference_counts(name):
    g = load_golden(f"trace_{name}.npz")
    parts, ex, ey, vac, p, bar = trace_args(g)
    got = OT.trace(*parts, ex, ey, vac, p, bar, rf=rf_of(g))
    np.testing.assert_array_equal(got[0], g["cnt_i"])
    np.testing.assert_array_equal(got[1], g["cnt_e"])
    np.testing.assert_array_equal(got[2], g["escaped"])
    assert got[3] == int(g["lost"])


@pytest.mark.parametrize("name", TRACE_CASES)
def test_oracle_record_matches_reference(name):
    g = load_golden(f"trace_{name}.npz")
    parts, ex, ey, vac, p, bar = trace_args(g)
    rec = {}
    got = OT.trace(*parts, ex, ey, vac, p, bar, record=rec, rf=rf_of(g))
    np.testing.assert_array_equal(got[0], g["rec_cnt_i"])
    np.testing.assert_array_equal(got[1], g["rec_cnt_e"])
    np.testing.assert_array_equal(rec["status"], g["rec_status"])
    np.testing.assert_array_equal(rec["hit_cells"], g["rec_hit_cells"])
    np.testing.assert_array_equal(rec["selected"], g["rec_selected"])
    tol = dict(rtol=1e-12, atol=1e-24) if rf_of(g) is not None else dict(rtol=0, atol=0)
    np.testing.assert_allclose(rec["endpoints"], g["rec_endpoints"], **tol)
    np.testing.assert_allclose(rec["final_velocity"], g["rec_final_velocity"], **tol)
    np.testing.assert_array_equal([len(v) for v in rec["paths"]], g["rec_path_lengths"])
    if len(rec["paths"]):
        np.testing.assert_allclose(np.concatenate(rec["paths"]), g["rec_paths"], **tol)
    if rf_of(g) is not None:
        np.testing.assert_allclose(rec["flight_time"], g["rec_flight_time"], rtol=1e-12, atol=1e-24)
        np.testing.assert_allclose(rec["final_phase"], g["rec_final_phase"], rtol=1e-12, atol=1e-9)


def test_oracle_is_independent_of_thread_count():
    g = load_golden("trace_cfg1.npz")
    parts, ex, ey, vac, p, bar = trace_args(g)
    a = OT.trace_detail(*parts[:5], ex, ey, vac, p, bar, threads=1)
    b = OT.trace_detail(*parts[:5], ex, ey, vac, p, bar, threads=7)
    for k in ("status", "hit", "steps", "x", "y", "vx", "vy"):
        np.testing.assert_array_equal(a[k], b[k])


@pytest.mark.parametrize("name", ["floating_leak", "floating_noleak", "fixed_leak", "dielectric_leak",
                                  "absorb_leak", "taper_leak", "base_noleak", "base_leak"])
def test_oracle_batch_loop_matches_reference_run(name):
    """Oracle batch loop + host geometry/injection == reference run() (bit for bit)."""
    g = load_golden(f"run_{name}.npz")
    p = g["p"]
    solid, mask, _, _ = geometry.build_geometry(p)
    np.testing.assert_array_equal(solid, g["solid"])
    np.testing.assert_array_equal(mask, g["mask"])
    st = OF.BatchState(p, solid, mask)
    rng = np.random.default_rng(p.seed)
    for _ in range(p.n_batches):
        x, y, vx, vy, qm, spc = inject.inject(p, p.n_per_batch, solid.shape[1], rng)
        st.step(*OT.trace(x, y, vx, vy, qm, spc, st.Ex, st.Ey, ~solid, p, st.barrier()))
    np.testing.assert_array_equal(st.rho, g["rho_raw"])
    np.testing.assert_allclose(st.phi, g["mean_phi"], rtol=0, atol=1e-12)
    for k in st.hist:
        np.testing.assert_array_equal(np.array(st.hist[k]), g[f"hist_{k}"])
    if "ref_data_rho" in g:
        # the reference's own regression data (tests/test_regression.py:41-50), made in its
        # origin environment: flux histories identical; charge and potential within the
        # rounding of another SciPy's sparse LU (the leakage operator is built from LU
        # solves), stated as 1e-13 of the charge scale and 1e-11 V
        np.testing.assert_array_equal(np.array(st.hist["ratio_i_bottom"]), g["ref_data_hist_ratio_i_bottom"])
        np.testing.assert_array_equal(np.array(st.hist["ratio_e_bottom"]), g["ref_data_hist_ratio_e_bottom"])
        ref_rho = g["ref_data_rho"]
        assert np.abs(st.rho - ref_rho).max() <= 1e-13 * np.abs(ref_rho).max()
        np.testing.assert_allclose(st.phi, g["ref_data_phi"], rtol=0, atol=1e-11)


def cfg1_ion_sampler(p):
    """DC 100 eV ions with polar angles N(0, 2 deg): the ion source of the 30-batch
    80x200 floating-mask fixture."""
    return inject.energy_angle_sampler(p, lambda r, k: np.full(k, 100.0), inject.gaussian_angle(2.0))


def test_oracle_batch_loop_matches_reference_cfg1_full_run():
    """80x200 floating conductive mask, 10k ions + 10k electrons per batch, 30 batches:
    the oracle batch loop reproduces the reference run() bit for bit."""
    g = load_golden("run_cfg1_30.npz")
    p = g["p"]
    solid, mask, _, _ = geometry.build_geometry(p)
    np.testing.assert_array_equal(solid, g["solid"])
    st = OF.BatchState(p, solid, mask)
    rng = np.random.default_rng(p.seed)
    samp = cfg1_ion_sampler(p)
    for _ in range(p.n_batches):
        parts = inject.inject(p, p.n_per_batch, solid.shape[1], rng, None, samp)
        st.step(*OT.trace(*parts, st.Ex, st.Ey, ~solid, p, st.barrier()))
    np.testing.assert_array_equal(st.rho, g["rho_raw"])
    np.testing.assert_allclose(st.phi, g["mean_phi"], rtol=0, atol=1e-12)
    for k in st.hist:
        np.testing.assert_array_equal(np.array(st.hist[k]), g[f"hist_{k}"])


@pytest.mark.parametrize("name", ["floating", "fixed", "dielectric", "cfg2"])
def test_oracle_fields_match_reference(name):
    g = load_golden(f"fields_{name}.npz")
    p = g["p"]
    f = OF.setup_fields(p, g["solid"], g["mask"])
    phi = f["solve"]((-g["rho"] / OF.EPS0).ravel()).reshape(g["solid"].shape) + f["external"]
    np.testing.assert_allclose(phi, g["phi"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(f["external"], g["external"], rtol=0, atol=1e-11)
    ex, ey = OF.compute_field(g["phi"], ~g["solid"], p)
    np.testing.assert_array_equal(ex, g["Ex"])
    np.testing.assert_array_equal(ey, g["Ey"])
    leak = OF.build_leakage(g["solid"], f["solve"], p)
    np.testing.assert_array_equal(leak["flat"], g["leak_flat"])
    np.testing.assert_array_equal(leak["region"], g["leak_region"])
    if "leak_M" in g:
        np.testing.assert_allclose(leak["M"], g["leak_M"], rtol=1e-9, atol=1e-12)
    else:
        q = np.random.default_rng(11).normal(size=(len(leak["flat"]), 4))
        np.testing.assert_allclose(leak["M"] @ q, g["leak_MQ"], rtol=1e-9, atol=1e-12)
    if "g_cond" in g:
        gc = OF.conductor_response(f["solve"], f["cond"], p.dx)
        np.testing.assert_allclose(gc, g["g_cond"], rtol=1e-10, atol=0)


def test_oracle_conductor_step_matches_reference():
    g = load_golden("conductor_step.npz")
    got = [OF.conductor_step(*a) for a in g["args"]]
    np.testing.assert_allclose(got, g["values"], rtol=1e-14, atol=0)


def circuit_of(g):
    return dict(t=g["circuit_t"], uw=g["circuit_uw"], um=g["circuit_um"], up=g["circuit_up"], V1=g["circuit_V1"])


def test_oracle_rf_batch_loop_matches_reference_run():
    """circuit_rf: RF basis, stratified launch phases and in-flight clock
    (trench_charging_2d.py:1079, 1231-1234) reproduce the reference run()."""
    g = load_golden("run_rf_taper.npz")
    p = g["p"]
    solid, mask, _, _ = geometry.build_geometry(p)
    st = OF.BatchState(p, solid, mask, circuit_of(g))
    rng = np.random.default_rng(p.seed)
    phase = np.random.default_rng(np.random.SeedSequence([p.seed, 0x5246]))
    period = st.fields["rf"]["period"]
    for _ in range(p.n_batches):
        parts = inject.inject(p, p.n_per_batch, solid.shape[1], rng, lambda r, k: np.full(k, p.electron_temp_eV / 2))
        rf = {**st.fields["rf"], "initial_time": np.concatenate(
            [inject.launch_times(phase, p.n_per_batch, period) for _ in range(2)])}
        st.step(*OT.trace(*parts, st.Ex, st.Ey, ~solid, p, st.barrier(), rf=rf))
    np.testing.assert_allclose(st.rho, g["rho_raw"], rtol=1e-12, atol=1e-6)
    np.testing.assert_allclose(st.phi, g["mean_phi"], rtol=0, atol=1e-9)
    for k in ("ratio_i_bottom", "ratio_e_bottom", "esc_e", "lost"):
        np.testing.assert_array_equal(np.array(st.hist[k]), g[f"hist_{k}"])
