"""Vertical-ion probe of a saturated charge state on the B200 tracer.

The reference's diagnostic (probe_vertical_ions, trench_charging_2d.py:1373-1439)
sends an equally spaced, exactly vertical ion beam of one energy across the
trench entrance and records it twice -- through the potential of the converged
charge and through the uncharged (external) potential -- leaving the charge as it
is.  ``VerticalProbe`` holds what the two traces share (the field solver, the beam,
the tracer, the RF launch phases) and traces one potential per call; recording
runs on the FP64 kernel, so hits, endpoints and paths follow the reference tracer.
``probe_vertical_ions`` is the reference-shaped entry point and returns the same
result dictionary.
"""
from dataclasses import fields as dc_fields
from dataclasses import replace

import numpy as np

from . import geometry
from .fields import compute_field, field_snapshot, setup_fields
from .inject import launch_times
from .params import AMU, E_CHARGE, EPS0, Params
from .tracer import B200Tracer

# settings that define the geometry, the boundaries and the ion species: the probe
# must share them with the run that produced the charge
RUN_SETTINGS = ("dx", "nx", "trench_w", "trench_offset", "trench_taper_deg", "trench_d", "floor_t", "n_vac",
                "mask_t", "mask_taper_deg", "mask_type", "eps_r", "mask_eps_r", "field_mode", "side_bc",
                "substrate_voltage", "mask_voltage", "top_voltage", "left_voltage", "right_voltage",
                "top_bc", "ion_mass_amu", "wall_model", "bias")


class VerticalProbe:
    """The probe of one converged run result (a dict with params, solid, mask, rho_raw,
    t_conv, stopped and, for circuit_rf, circuit)."""

    def __init__(self, res, p=None, phase=None, device=0):
        if res.get("stopped", False) or not np.isfinite(res.get("t_conv", np.nan)):
            raise ValueError("the probe needs a run result that passed the steady-state check")
        known = {f.name for f in dc_fields(Params)}
        run_p = Params(**{k: v for k, v in dict(res["params"]).items() if k in known})
        p = run_p if p is None else p
        changed = [k for k in RUN_SETTINGS if getattr(p, k) != getattr(run_p, k)]
        if changed:
            raise ValueError(f"the probe must keep the charging run's geometry and boundaries ({', '.join(changed)})")
        if not (1 <= p.probe_trajectories <= p.probe_ions and np.isfinite(p.probe_energy_eV)
                and p.probe_energy_eV > 0):
            raise ValueError("the probe needs probe_ions >= probe_trajectories >= 1 and a positive energy")
        self.p = p if phase is None else replace(p, rf_phase=phase)
        self.res = res
        self.solid = np.asarray(res["solid"])
        self.vac = ~self.solid
        self.fields = setup_fields(self.p, self.solid, np.asarray(res["mask"]), res.get("circuit"), device=device)
        self.tracer = B200Tracer(self.vac, device)
        self.wface = np.where(self.fields["cond"], 1.0, self.fields["eps"] / (1 + self.fields["eps"]))
        q = self.p
        self.entrance = geometry.opening_span(self.solid, q.floor_t + q.trench_d + q.mask_t - 1)
        self.bottom = geometry.opening_span(self.solid, q.floor_t)
        self.beam = self._beam()
        self.rf = None
        if self.fields["rf"] is not None:
            # launch phases spread over the period, seeded from the run's seed
            rng = np.random.default_rng(np.random.SeedSequence([q.seed, 0x50524F42]))
            period = self.fields["rf"]["period"]
            self.rf = {**self.fields["rf"], "initial_time": launch_times(rng, q.probe_ions, period)}

    def _beam(self):
        """probe_ions ions at the mid-points of equal slices of the entrance opening, one
        cell fraction below the top, moving straight down at the probe energy."""
        q = self.p
        e0, e1 = self.entrance
        k = q.probe_ions
        mass = q.ion_mass_amu * AMU
        x = (e0 + (np.arange(k) + 0.5) * (e1 - e0) / k) * q.dx
        return dict(x=x, y=np.full(k, (self.solid.shape[1] - 1e-3) * q.dx), vx=np.zeros(k),
                    vy=np.full(k, -np.sqrt(2 * q.probe_energy_eV * E_CHARGE / mass)),
                    qm=np.full(k, E_CHARGE / mass), spc=np.zeros(k, dtype=np.int8))

    def charged_potential(self):
        rho = np.asarray(self.res["rho_raw"])
        return self.fields["solve"]((-rho / EPS0).ravel()).reshape(self.solid.shape) + self.fields["external"]

    def trace(self, phi, stop=None):
        """Record the beam through potential `phi`; returns the reference's record dict
        for one potential (hits, paths, endpoints, impact angles and energies, the
        bottom fraction and flux, the displayed potential and field)."""
        q, b = self.p, self.beam
        ex, ey = compute_field(phi, self.vac, q, self.fields["volts"]["top"])
        barrier = (phi, self.wface) if q.wall_model == "barrier" else None
        rec = {}
        ci, _, esc, lost = self.tracer(*(b[k].copy() for k in ("x", "y", "vx", "vy", "qm", "spc")), ex, ey, self.vac,
                                       q, barrier, record=rec, stop=stop, rf=self.rf)
        shown, _, _, volts = field_snapshot(self.fields, phi, q)
        shown_ex, shown_ey = compute_field(shown, self.vac, q, volts["top"])
        b0, b1 = self.bottom
        e0, e1 = self.entrance
        floor_hits = ci[b0:b1, q.floor_t - 1]
        v_end = rec["final_velocity"]
        rec.update(phi=shown, Ex=shown_ex, Ey=shown_ey, hits=ci, escaped=int(esc[0]), lost=lost,
                   bottom_fraction=float(floor_hits.sum() / q.probe_ions),
                   bottom_flux=floor_hits * q.flux * (e1 - e0) / q.probe_ions,
                   angle_deg=np.degrees(np.arctan2(v_end[:, 0], -v_end[:, 1])),
                   impact_energy_eV=q.ion_mass_amu * AMU / (2 * E_CHARGE) * np.sum(v_end ** 2, axis=1))
        return rec


def probe_vertical_ions(res, p=None, phase=None, log=print, stop=None, device=0):
    """The reference-shaped probe call: the result dict with a 'charged' and an
    'uncharged' record (the second is skipped when a stop request cancels the first)."""
    probe = VerticalProbe(res, p, phase, device)
    q = probe.p
    (e0, e1), (b0, b1) = probe.entrance, probe.bottom
    out = dict(energy_eV=q.probe_energy_eV, n_ions=q.probe_ions, phase=q.rf_phase, entrance_i0=e0, entrance_i1=e1,
               bottom_i0=b0, bottom_i1=b1, source_t_conv=res["t_conv"], source_converged=True, cancelled=False,
               backend_used="b200", rf_cycle=probe.rf is not None)
    if probe.rf is not None:
        out.update(rf_period=probe.rf["period"], rf_time_steps=q.rf_time_steps)
    for label, phi in (("charged", probe.charged_potential()), ("uncharged", probe.fields["external"])):
        if log is not None:
            log(f"vertical-ion probe: {label}, {q.probe_ions} ions, {q.probe_energy_eV:g} eV")
        out[label] = probe.trace(phi, stop)
        if out[label]["cancelled"]:
            out["cancelled"] = True
            break
    return out
