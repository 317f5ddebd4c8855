"""Generates the golden fixtures in this folder by running the reference here.

    python tests/golden/make_golden.py /path/to/reference
    (or TRENCH01_REFERENCE=/path/to/reference python tests/golden/make_golden.py)

The reference (a Python package) is imported from its source tree with a stub
``matplotlib`` (only ``use`` and an empty ``pyplot`` are needed on the compute
path).  Every fixture stores the reference's inputs and outputs, so tests check
the oracle and the CUDA path without the reference present.

Fixtures:
  trace_*.npz   tracer inputs (particles, fields, barrier) and trace_cpu outputs
                (trench_charging_2d.py:542-702), with per-particle record data
  run_*.npz     short run() batch loops: rho_raw, mean_phi, history
                (trench_charging_2d.py:1045-1369)
  fields_*.npz  setup_fields / solve / compute_field / build_leakage /
                conductor_response outputs for one geometry
  steady_checks.npz  the steady-state check functions on seeded synthetic histories
                (trench_charging_2d.py:877-945)
  steady_run_*.npz  run() with until_steady to convergence: histories, charge
                monitors, convergence batch
  regression_pin.json  agreement of run() here with the reference's own
                tests/data/*.npz (tests/test_regression.py:41-50)
"""
import json
import sys
import tempfile
import types
from dataclasses import asdict, replace
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def reference_dir(argv):
    """The reference's source tree: the first argument, else $TRENCH01_REFERENCE."""
    import os
    ref = argv[1] if len(argv) > 1 else os.environ.get("TRENCH01_REFERENCE")
    if not ref:
        raise SystemExit("name the reference's source tree: make_golden.py PATH or TRENCH01_REFERENCE=PATH")
    return ref


def import_reference(path):
    stub = Path(tempfile.mkdtemp()) / "matplotlib"
    stub.mkdir()
    (stub / "__init__.py").write_text("def use(*a, **k):\n    pass\n")
    (stub / "pyplot.py").write_text("")
    sys.path.insert(0, str(stub.parent))
    sys.path.insert(0, str(path))
    import trench_charging_2d as T
    import trench_rf as RF
    return T, RF


def params_json(p):
    return json.dumps(asdict(p))


def save(name, **arrays):
    np.savez_compressed(OUT / name, **arrays)
    size = (OUT / name).stat().st_size
    print(f"wrote {name} ({size/1024:.0f} KiB)")


def trace_case(T, name, p, phi, fields, solid, seed, n, barrier=True, rf=None, ion_energy=None, rng=None):
    ex, ey = T.compute_field(phi, ~solid, p, fields["volts"]["top"])
    wface = np.where(fields["cond"], 1.0, fields["eps"] / (1 + fields["eps"]))
    rng = rng if rng is not None else np.random.default_rng(seed)
    parts = T.inject(p, n, solid.shape[1], rng, ion_energy)
    bar = (phi, wface) if barrier else None
    out = {}
    for rec in (False, True):
        record = {} if rec else None
        res = T.trace_cpu(*(v.copy() for v in parts), ex, ey, ~solid, p, bar, record, rf=rf)
        if not rec:
            out.update(cnt_i=res[0], cnt_e=res[1], escaped=res[2], lost=np.int64(res[3]))
        else:
            out.update(rec_cnt_i=res[0], rec_cnt_e=res[1], rec_escaped=res[2], rec_lost=np.int64(res[3]),
                       rec_status=record["status"], rec_hit_cells=record["hit_cells"],
                       rec_endpoints=record["endpoints"], rec_final_velocity=record["final_velocity"],
                       rec_selected=record["selected"],
                       rec_path_lengths=np.array([len(v) for v in record["paths"]]),
                       rec_paths=np.concatenate(record["paths"]) if record["paths"] else np.zeros((0, 2)))
            if rf is not None:
                out.update(rec_flight_time=record["flight_time"], rec_final_phase=record["final_phase"])
    extra = {}
    if rf is not None:
        extra = dict(rf_period=rf["period"], rf_dt_max=rf["dt_max"], rf_wave=rf["wave"], rf_phi=rf["phi"],
                     rf_Ex=rf["Ex"], rf_Ey=rf["Ey"], rf_initial_time=rf["initial_time"])
    x, y, vx, vy, qm, spc = parts
    save(f"trace_{name}.npz", params=params_json(p), solid=solid, x=x, y=y, vx=vx, vy=vy, qm=qm, spc=spc,
         Ex=ex, Ey=ey, phi=phi, wface=wface, barrier=np.bool_(barrier), **out, **extra)


def charged_state(T, p, n_batches):
    """Reference run() for a few batches; returns its charged potential."""
    res = T.run(replace(p, n_batches=n_batches), log=lambda s: None)
    return res["mean_phi"], res


def main(ref):
    T, RF = import_reference(ref)
    P = T.Params

    # --- tracer cases -------------------------------------------------------
    small = replace(P(), nx=30, trench_w=10, trench_d=20, floor_t=5, mask_t=6, n_vac=12, bias="dc", sigma_s=0,
                    n_batches=8, n_per_batch=400, max_steps=1000, probe_trajectories=12)
    solid, mask, i0, i1 = T.build_geometry(small)
    f = T.setup_fields(small, solid, mask)
    rho = np.zeros(solid.shape)
    rho[i0 - 1, small.floor_t:small.floor_t + small.trench_d] = 2e7
    rho[i1, small.floor_t:small.floor_t + small.trench_d] = -1e7
    phi = f["solve"]((-rho / T.EPS0).ravel()).reshape(solid.shape)
    for wall in ("barrier", "absorb"):
        trace_case(T, f"small_{wall}", replace(small, wall_model=wall), phi, f, solid, 20, 400,
                   barrier=wall == "barrier")

    tr, ma = np.degrees(np.arctan(.25)), np.degrees(np.arctan(.5))
    taper = replace(P(), nx=40, trench_w=16, trench_d=20, floor_t=4, mask_t=12, n_vac=10, trench_taper_deg=tr,
                    mask_taper_deg=ma, bias="dc", sigma_s=0, n_per_batch=256, max_steps=800,
                    field_mode="fixed", substrate_voltage=-30, mask_voltage=-10, probe_trajectories=12)
    solid, mask, i0, i1 = T.build_geometry(taper)
    f = T.setup_fields(taper, solid, mask)
    regions = T.charge_monitors(solid, mask, i0, i1, taper)
    rho = np.zeros(solid.shape)
    rho.ravel()[regions["left"]] = 2e6
    rho.ravel()[regions["right"]] = -1e6
    phi = f["solve"]((-rho / T.EPS0).ravel()).reshape(solid.shape) + f["external"]
    for wall in ("barrier", "absorb"):
        trace_case(T, f"taper_{wall}", replace(taper, wall_model=wall), phi, f, solid, 22, 256,
                   barrier=wall == "barrier")

    # Configuration-1 geometry (80x200, conductive floating mask), charged by 6 batches.
    cfg1 = replace(P(), dx=5e-9, nx=80, trench_w=20, trench_d=60, floor_t=20, mask_t=20, n_vac=100,
                   mask_type="conductor", field_mode="floating", sigma_s=1e-15, wall_model="barrier", bias="dc",
                   ion_energy_eV=100, electron_temp_eV=4, n_per_batch=2000, seed=0, probe_trajectories=16)
    phi, _ = charged_state(T, cfg1, 6)
    solid, mask, _, _ = T.build_geometry(cfg1)
    f = T.setup_fields(cfg1, solid, mask)
    trace_case(T, "cfg1", cfg1, phi, f, solid, 100, 2000)

    # Configuration-2 geometry (60x250 AR 8, tapers 2/5 deg, dielectric mask), charged by 6 batches.
    cfg2 = replace(P(), nx=60, trench_w=20, trench_d=160, floor_t=10, mask_t=20, n_vac=60, trench_taper_deg=2.0,
                   mask_taper_deg=5.0, mask_type="dielectric", mask_eps_r=3.0, electron_temp_eV=3.0, bias="dc",
                   ion_energy_eV=90.0, n_per_batch=2000, seed=1, probe_trajectories=16)
    phi, _ = charged_state(T, cfg2, 6)
    solid, mask, _, _ = T.build_geometry(cfg2)
    f = T.setup_fields(cfg2, solid, mask)
    trace_case(T, "cfg2", cfg2, phi, f, solid, 101, 2000)

    # RF in-flight clock on a tapered trench (test_taper.py:273-294 waveform).
    rfp = replace(taper, bias="rf", field_mode="circuit_rf", side_bc="pillar", rf_freq=5e8)
    t = np.arange(256) / 256 / rfp.rf_freq
    c = dict(t=t, uw=-60 - 20 * np.sin(2 * np.pi * t * rfp.rf_freq), um=-30 - 10 * np.sin(2 * np.pi * t * rfp.rf_freq),
             up=t * 0, V1=30 + 10 * np.sin(2 * np.pi * t * rfp.rf_freq))
    solid, mask, _, _ = T.build_geometry(rfp)
    f = T.setup_fields(rfp, solid, mask, c)
    rng = np.random.default_rng(3)
    n = 512
    parts_rng = np.random.default_rng(3)
    rf = {**f["rf"], "initial_time": np.concatenate([RF.launch_times(np.random.default_rng(4), n, f["rf"]["period"])
                                                     for _ in range(2)])}
    trace_case(T, "rf_taper", rfp, f["external"], f, solid, 3, n, rf=rf,
               ion_energy=lambda r, k: np.full(k, rfp.electron_temp_eV / 2), rng=parts_rng)
    del rng

    # --- batch-loop runs ----------------------------------------------------
    base = dict(nx=30, trench_w=10, trench_d=20, floor_t=5, mask_t=6, n_vac=12, bias="dc", n_per_batch=400,
                max_steps=1000, n_batches=4)
    runs = {
        "floating_leak": replace(P(), sigma_s=1e-14, **base),
        "floating_noleak": replace(P(), sigma_s=0.0, **base),
        "fixed_leak": replace(P(), sigma_s=1e-14, field_mode="fixed", substrate_voltage=-20, mask_voltage=-10,
                              **base),
        "dielectric_leak": replace(P(), sigma_s=1e-14, mask_type="dielectric", **base),
        "absorb_leak": replace(P(), sigma_s=1e-14, wall_model="absorb", **base),
        "taper_leak": replace(P(), nx=40, trench_w=16, trench_d=20, floor_t=4, mask_t=12, n_vac=10,
                              trench_taper_deg=tr, mask_taper_deg=ma, bias="dc", sigma_s=1e-14, n_per_batch=256,
                              max_steps=800, n_batches=3),
    }
    display = lambda res: dict(rho_display=res["rho"], phi_display=res["phi"], external_phi=res["external_phi"],
                               Ex_display=res["Ex"], Ey_display=res["Ey"],
                               volts=np.array([res["voltages"][k] for k in ("substrate", "mask", "top")]))
    for name, p in runs.items():
        res = T.run(p, log=lambda s: None)
        save(f"run_{name}.npz", params=params_json(p), rho_raw=res["rho_raw"], mean_phi=res["mean_phi"],
             solid=res["solid"], mask=res["mask"], **display(res),
             **{f"hist_{k}": np.asarray(v) for k, v in res["hist"].items()})

    # circuit_rf batch loop with the reference's test waveform (tests/test_taper.py:273-283)
    rfrun = replace(taper, bias="rf", field_mode="circuit_rf", side_bc="pillar", rf_freq=5e8, sigma_s=1e-14,
                    n_batches=3, wall_model="barrier")
    tt = np.arange(256) / 256 / rfrun.rf_freq
    circ = dict(t=tt, uw=-60 - 20 * np.sin(2 * np.pi * tt * rfrun.rf_freq),
                um=-30 - 10 * np.sin(2 * np.pi * tt * rfrun.rf_freq), up=tt * 0,
                V1=30 + 10 * np.sin(2 * np.pi * tt * rfrun.rf_freq), E=np.array([]),
                us=-60 - 20 * np.sin(2 * np.pi * tt * rfrun.rf_freq), i=tt * 0, cached=False, ied_model="instant",
                sheath=None, n_periods=1, elements={}, ied_computed=False, s=1e-5, tau_i=1e-9)
    import copy
    orig_solve, orig_summary = T.PC.solve_circuit_cached, T.PC.summary
    T.PC.solve_circuit_cached = lambda *a, **k: copy.deepcopy(circ)
    T.PC.summary = lambda c: "test circuit"
    try:
        res = T.run(rfrun, log=lambda s: None)
    finally:
        T.PC.solve_circuit_cached, T.PC.summary = orig_solve, orig_summary
    save("run_rf_taper.npz", params=params_json(rfrun), rho_raw=res["rho_raw"], mean_phi=res["mean_phi"],
         solid=res["solid"], mask=res["mask"], circuit_t=circ["t"], circuit_uw=circ["uw"], circuit_um=circ["um"],
         circuit_up=circ["up"], circuit_V1=circ["V1"], **display(res),
         **{f"hist_{k}": np.asarray(v) for k, v in res["hist"].items()})

    # --- vertical-ion probe (trench_charging_2d.py:1373-1439) -------------------
    def probe_case(name, p, rho):
        solid, mask, i0, i1 = T.build_geometry(p)
        res = dict(params=asdict(p), solid=solid, mask=mask, i0=i0, i1=i1, rho_raw=rho, t_conv=1e-3,
                   stopped=False, circuit=None)
        out = T.probe_vertical_ions(res, log=lambda s: None)
        arrays = {}
        for label in ("charged", "uncharged"):
            r = out[label]
            for k in ("hits", "status", "hit_cells", "endpoints", "final_velocity", "angle_deg",
                      "impact_energy_eV", "bottom_flux", "phi", "Ex", "Ey"):
                arrays[f"{label}_{k}"] = np.asarray(r[k])
            arrays[f"{label}_scalars"] = np.array([r["bottom_fraction"], r["escaped"], r["lost"]], dtype=float)
            arrays[f"{label}_path_lengths"] = np.array([len(v) for v in r["paths"]])
            arrays[f"{label}_paths"] = np.concatenate(r["paths"])
        save(f"probe_{name}.npz", params=params_json(p), solid=solid, mask=mask, rho_raw=rho, **arrays)

    pt = replace(taper, field_mode="floating", substrate_voltage=0, mask_voltage=0, probe_ions=224,
                 probe_trajectories=12)
    probe_case("taper_empty", pt, np.zeros(T.build_geometry(pt)[0].shape))
    ps = replace(P(), nx=20, trench_w=6, trench_d=12, floor_t=4, mask_t=4, n_vac=8, bias="dc", sigma_s=0,
                 probe_ions=120, probe_trajectories=8, max_steps=800)
    solid, mask, i0, i1 = T.build_geometry(ps)
    rho = np.zeros(solid.shape)
    rho[i0 - 1, ps.floor_t:ps.floor_t + ps.trench_d] = 1e7
    probe_case("small_charged", ps, rho)

    # --- field-side cases -----------------------------------------------------
    for name, p in {"floating": runs["floating_leak"], "fixed": runs["fixed_leak"],
                    "dielectric": runs["dielectric_leak"],
                    "cfg2": replace(cfg2, sigma_s=1e-15)}.items():
        solid, mask, i0, i1 = T.build_geometry(p)
        f = T.setup_fields(p, solid, mask)
        rng = np.random.default_rng(7)
        rho = np.zeros(solid.shape)
        surf = T.surface_cells(solid)
        rho[surf] = rng.normal(0, 3e6, surf.sum())
        if f["cond"].any():
            rho[f["cond"]] = 0.0
            c_cell = np.flatnonzero(surf & f["cond"])[0]
            rho.flat[c_cell] = 5e6
        phi = f["solve"]((-rho / T.EPS0).ravel()).reshape(solid.shape) + f["external"]
        ex, ey = T.compute_field(phi, ~solid, p, f["volts"]["top"])
        leak = T.build_leakage(solid, f["solve"], i0, i1, p)
        extra = {}
        if f["floating"]:
            g = T.conductor_response(f["solve"], f["cond"], p.dx)
            extra = dict(g_cond=g, C_cond=1.0 / g[f["cond"]][0])
        m = len(leak["flat"])
        if m <= 200:
            extra["leak_M"] = leak["M"]
        else:
            # Large operators are pinned through their action on seeded vectors.
            extra["leak_MQ"] = leak["M"] @ np.random.default_rng(11).normal(size=(m, 4))
        save(f"fields_{name}.npz", params=params_json(p), solid=solid, mask=mask, rho=rho, phi=phi, Ex=ex, Ey=ey,
             external=f["external"], leak_flat=leak["flat"], leak_region=leak["region"], **extra)

    # conductor_step values (trench_charging_2d.py:815-830)
    cases = [(120, 80, 3e-12, 2e-10, 3.0, 0.0), (0, 50, 1e-12, 1e-10, 4.0, 0.01), (40, 0, 1e-12, 1e-10, 4.0, -0.2),
             (500, 500, 2e-12, 3e-10, 3.0, 0.05), (10, 900, 1e-12, 1e-10, 2.0, 0.0)]
    vals = [T.conductor_step(*c) for c in cases]
    save("conductor_step.npz", args=np.array(cases, dtype=float), values=np.array(vals))

    # --- configuration 1, full run (30 batches, 10k ions + 10k electrons, DC 100 eV, angles N(0, 2 deg)) ----
    sys.path.insert(0, str(OUT.parents[1]))
    from trench_b200 import inject as b200_inject
    cfg1_run = replace(cfg1, n_per_batch=10000, n_batches=30, probe_trajectories=40)
    sampler = b200_inject.energy_angle_sampler(cfg1_run, lambda r, k: np.full(k, 100.0),
                                               b200_inject.gaussian_angle(2.0))
    orig_inject = T.inject
    T.inject = lambda p_, n_, ny_, rng_, ie=None, iv=None: orig_inject(p_, n_, ny_, rng_, None, sampler)
    try:
        res = T.run(cfg1_run, log=lambda s: None)
    finally:
        T.inject = orig_inject
    save("run_cfg1_30.npz", params=params_json(cfg1_run), rho_raw=res["rho_raw"], mean_phi=res["mean_phi"],
         solid=res["solid"], mask=res["mask"], **{f"hist_{k}": np.asarray(v) for k, v in res["hist"].items()})

    # --- steady-state stopping (until_steady) -----------------------------------
    # the check functions on seeded synthetic histories (trench_charging_2d.py:877-945)
    rs = np.random.default_rng(77)
    series = []
    for k in range(12):
        n = 30
        t = np.arange(n)
        x = rs.normal(0, 1 + k % 3, n) + (0.05 * k) * t
        if k % 4 == 3:
            x = np.cumsum(x) * 0.1   # strongly autocorrelated
        series.append(x)
    series = np.array(series)
    mse = np.array([T._mean_and_se(x) for x in series])
    sp = replace(P(), steady_window=15, steady_rtol=0.005, steady_charge_rtol=0.005, steady_charge_atol=1e-15,
                 dt_batch=1e-4)
    probe_names = ["a", "b", "c"]
    vcases, ccases = [], []
    for k in range(6):
        h = {nm: list(20 + rs.normal(0, 0.05, 30) + (0.02 * k * (j + 1)) * np.arange(30) / 30)
             for j, nm in enumerate(probe_names)}
        ok, name, d, tol = T.check_steady(h, probe_names, sp, None)
        vcases.append(([h[nm] for nm in probe_names], [float(ok), probe_names.index(name), d, tol]))
        q = {nm: list(1e-12 * (1 + rs.normal(0, 0.01, 30) + 0.01 * k * np.arange(30) / 30))
             for nm in ("left", "right")}
        c = T.check_charge_steady(q, sp)
        ccases.append(([q["left"], q["right"]],
                       [float(c["ok"]), ["left", "right"].index(c["name"]), float(c["kind"] == "drift"),
                        c["d"], c["tol"], c["ratio"], c["rate"]]))
    save("steady_checks.npz", params=params_json(sp), series=series, mean_se=mse,
         v_hist=np.array([v[0] for v in vcases]), v_out=np.array([v[1] for v in vcases]),
         q_hist=np.array([c[0] for c in ccases]), q_out=np.array([c[1] for c in ccases]))
    # whole runs to steady charge
    steady_runs = {
        "floating": replace(P(), sigma_s=1e-14, until_steady=True, max_batches=400, steady_window=5, steady_hold=2,
                            **{k: v for k, v in base.items() if k != "n_batches"}),
        "dielectric": replace(P(), sigma_s=1e-14, mask_type="dielectric", until_steady=True, max_batches=400,
                              steady_window=10, steady_hold=2, **{k: v for k, v in base.items() if k != "n_batches"}),
    }
    for name, p in steady_runs.items():
        res = T.run(p, log=lambda s: None)
        save(f"steady_run_{name}.npz", params=params_json(p), rho_raw=res["rho_raw"], mean_phi=res["mean_phi"],
             converged=np.array(res["converged"]), t_conv=np.array(res["t_conv"]),
             steady_n_ok=np.array(res["checkpoint"]["steady_n_ok"]),
             steady_names=np.array(list(res["steady"])), steady_values=np.array(list(res["steady"].values())),
             **{f"hist_{k}": np.asarray(v) for k, v in res["hist"].items()},
             **{f"charge_{k}": np.asarray(v) for k, v in res["charge_hist"].items()},
             **{f"monitor_{k}": np.asarray(v) for k, v in res["charge_monitor_hist"].items()})

    # --- agreement with the reference's own regression data -------------------
    pin = {}
    data = Path(ref) / "tests" / "data"
    for name, sigma in (("base_noleak", 0.0), ("base_leak", 1e-14)):
        p = replace(P(), mask_t=0, n_batches=40, bias="dc", sigma_s=sigma, wall_model="absorb")
        res = T.run(p, log=lambda s: None)
        with np.load(data / f"{name}.npz") as d:
            pin[name] = dict(
                rho_max_abs_diff=float(np.max(np.abs(d["rho"] - res["rho"]))),
                phi_max_abs_diff=float(np.max(np.abs(d["phi"] - res["phi"]))),
                hist_ratio_i_equal=bool(np.array_equal(d["hist_ratio_i_bottom"], res["hist"]["ratio_i_bottom"])),
                hist_ratio_e_equal=bool(np.array_equal(d["hist_ratio_e_bottom"], res["hist"]["ratio_e_bottom"])))
            save(f"run_{name}.npz", params=params_json(p), rho_raw=res["rho_raw"], mean_phi=res["mean_phi"],
                 solid=res["solid"], mask=res["mask"], ref_data_rho=d["rho"], ref_data_phi=d["phi"],
                 ref_data_hist_ratio_i_bottom=d["hist_ratio_i_bottom"],
                 ref_data_hist_ratio_e_bottom=d["hist_ratio_e_bottom"],
                 **{f"hist_{k}": np.asarray(v) for k, v in res["hist"].items()})
    (OUT / "regression_pin.json").write_text(json.dumps(pin, indent=1) + "\n")
    print(json.dumps(pin, indent=1))


if __name__ == "__main__":
    main(reference_dir(sys.argv))
