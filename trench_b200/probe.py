"""Vertical-ion probe of a saturated charge state on the B200 tracer.

Restates probe_vertical_ions (trench_charging_2d.py:1373-1439): an equally spaced,
exactly vertical ion beam over the entrance, traced with trajectory recording
through the charged and the uncharged potential, without changing the charge.
Recording runs on the FP64 kernel, so hits, endpoints and paths follow the
reference tracer.
"""
from dataclasses import fields as dc_fields
from dataclasses import replace

import numpy as np

from . import geometry
from .fields import compute_field, field_snapshot, setup_fields
from .inject import launch_times
from .params import AMU, E_CHARGE, EPS0, Params
from .tracer import B200Tracer

SAME_SETTINGS = ("dx", "nx", "trench_w", "trench_offset", "trench_taper_deg", "trench_d", "floor_t", "n_vac",
                 "mask_t", "mask_taper_deg", "mask_type", "eps_r", "mask_eps_r", "field_mode", "side_bc",
                 "substrate_voltage", "mask_voltage", "top_voltage", "left_voltage", "right_voltage",
                 "top_bc", "ion_mass_amu", "wall_model", "bias")


def _params(d):
    names = {f.name for f in dc_fields(Params)}
    return Params(**{k: v for k, v in dict(d).items() if k in names})


def probe_vertical_ions(res, p=None, phase=None, log=print, stop=None, device=0):
    """res: a run result with params, solid, mask, rho_raw, t_conv, stopped and (for RF)
    circuit; returns the reference's result dict with 'charged' and 'uncharged' records."""
    if not np.isfinite(res.get("t_conv", np.nan)) or res.get("stopped", False):
        raise ValueError("the probe needs a result that passed the steady-state check")
    source = _params(res["params"])
    p = source if p is None else p
    for key in SAME_SETTINGS:
        if getattr(p, key) != getattr(source, key):
            raise ValueError("the probe must use the geometry and boundary settings of the charging run")
    if (p.probe_ions < 1 or p.probe_trajectories < 1 or p.probe_trajectories > p.probe_ions
            or not np.isfinite(p.probe_energy_eV) or p.probe_energy_eV <= 0):
        raise ValueError("probe ion count and energy must be positive, trajectories <= ions")
    if phase is not None:
        p = replace(p, rf_phase=phase)
    solid, mask = np.asarray(res["solid"]), np.asarray(res["mask"])
    vac = ~solid
    fields = setup_fields(p, solid, mask, res.get("circuit"), device=device)
    tracer = B200Tracer(vac, device)
    ny = solid.shape[1]
    i0, i1 = geometry.opening_span(solid, p.floor_t + p.trench_d + p.mask_t - 1)
    b0, b1 = geometry.opening_span(solid, p.floor_t)
    x = (i0 + (np.arange(p.probe_ions) + 0.5) * (i1 - i0) / p.probe_ions) * p.dx
    y = np.full(x.size, (ny - 1e-3) * p.dx)
    vx = np.zeros(x.size)
    vy = np.full(x.size, -np.sqrt(2 * p.probe_energy_eV * E_CHARGE / (p.ion_mass_amu * AMU)))
    qm = np.full(x.size, E_CHARGE / (p.ion_mass_amu * AMU))
    spc = np.zeros(x.size, dtype=np.int8)
    charged_phi = fields["solve"]((-np.asarray(res["rho_raw"]) / EPS0).ravel()).reshape(solid.shape) \
        + fields["external"]
    wface = np.where(fields["cond"], 1.0, fields["eps"] / (1 + fields["eps"]))
    result = dict(energy_eV=p.probe_energy_eV, n_ions=x.size, phase=p.rf_phase, entrance_i0=i0, entrance_i1=i1,
                  bottom_i0=b0, bottom_i1=b1, source_t_conv=res["t_conv"], source_converged=True, cancelled=False,
                  backend_used="b200", rf_cycle=fields["rf"] is not None)
    options = {}
    if fields["rf"] is not None:
        rng = np.random.default_rng(np.random.SeedSequence([p.seed, 0x50524F42]))
        options["rf"] = {**fields["rf"], "initial_time": launch_times(rng, x.size, fields["rf"]["period"])}
        result["rf_period"] = fields["rf"]["period"]
        result["rf_time_steps"] = p.rf_time_steps
    for label, phi in (("charged", charged_phi), ("uncharged", fields["external"])):
        if log is not None:
            log(f"vertical-ion probe: {label}, {x.size} ions, {p.probe_energy_eV:g} eV")
        Ex, Ey = compute_field(phi, vac, p, fields["volts"]["top"])
        record = {}
        ci, _, esc, lost = tracer(x.copy(), y.copy(), vx.copy(), vy.copy(), qm.copy(), spc.copy(), Ex, Ey, vac, p,
                                  (phi, wface) if p.wall_model == "barrier" else None, record=record, stop=stop,
                                  **options)
        shown_phi, _, _, volts = field_snapshot(fields, phi, p)
        shown_ex, shown_ey = compute_field(shown_phi, vac, p, volts["top"])
        record.update(phi=shown_phi, Ex=shown_ex, Ey=shown_ey, hits=ci, escaped=int(esc[0]), lost=lost,
                      bottom_fraction=float(ci[b0:b1, p.floor_t - 1].sum() / x.size),
                      bottom_flux=ci[b0:b1, p.floor_t - 1] * p.flux * (i1 - i0) / x.size)
        record["angle_deg"] = np.degrees(np.arctan2(record["final_velocity"][:, 0], -record["final_velocity"][:, 1]))
        record["impact_energy_eV"] = (p.ion_mass_amu * AMU / (2 * E_CHARGE)
                                      * np.sum(record["final_velocity"] ** 2, axis=1))
        result[label] = record
        if record["cancelled"]:
            result["cancelled"] = True
            return result
    return result
