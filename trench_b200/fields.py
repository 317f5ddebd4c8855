"""Poisson operator, boundary potentials and the multigrid solver on the device.

Host-side assembly (once per case) restates the reference's operator and
boundary terms; the solve runs on the GPU through ``tb_poisson_setup`` /
``tb_poisson_solve`` (multigrid-preconditioned CG, FP32 V-cycles, FP64
refinement).  ``FieldSolver.solve`` is a drop-in for the reference's
``fields["solve"]`` (trench_charging_2d.py:297-309, 378-392): it takes the
right-hand side b of A phi = b (flat, or column-stacked), and returns phi with
the same conductor semantics (floating conductor as one unknown, driven
conductor held at zero).
"""
import ctypes

import numpy as np
import torch

from . import _capi
from .params import EPS0, FIELD_MODES, SIDE_BCS


def poisson_matrix_arrays(eps, cond, p):
    """Diagonal and east/north face coefficients of div(eps grad) (trench_charging_2d.py:252-294).

    Returns (diag, ce, cn) with A phi = diag*phi + ce*phi_E + cw*phi_W + cn*phi_N + cs*phi_S,
    cw = roll(ce, 1), cs[:, 1:] = cn[:, :-1]; cn[:, -1] = 0.
    """
    nx, ny = eps.shape
    dx2 = p.dx ** 2

    def face(a, b, ca, cb):
        h = np.where(ca, 2.0 * b, np.where(cb, 2.0 * a, 2.0 * a * b / (a + b)))
        return np.where(ca & cb, 0.0, h)

    ce = face(eps, np.roll(eps, -1, axis=0), cond, np.roll(cond, -1, axis=0)) / dx2
    top_ox = p.floor_t + p.trench_d
    if p.side_bc != "periodic":
        ce[-1, :top_ox] = 0.0
    cw = np.roll(ce, 1, axis=0)
    c_int = face(eps[:, :-1], eps[:, 1:], cond[:, :-1], cond[:, 1:]) / dx2
    cn = np.zeros((nx, ny)); cn[:, :-1] = c_int
    cs = np.zeros((nx, ny)); cs[:, 1:] = c_int
    diag_n, diag_s = cn.copy(), cs.copy()
    diag_s[:, 0] += 2.0 * eps[:, 0] / dx2
    if p.top_bc == "dirichlet":
        diag_n[:, -1] += 2.0 * eps[:, -1] / dx2
    diag = -(ce + cw + diag_n + diag_s)
    if p.side_bc != "periodic":
        diag[0, :top_ox] -= 2.0 * eps[0, :top_ox] / dx2
        diag[-1, :top_ox] -= 2.0 * eps[-1, :top_ox] / dx2
    return diag, ce, cn


def apply_matrix(diag, ce, cn, phi):
    """A @ phi for the arrays of poisson_matrix_arrays (phi shaped (nx, ny))."""
    out = diag * phi + ce * np.roll(phi, -1, axis=0) + np.roll(ce, 1, axis=0) * np.roll(phi, 1, axis=0)
    out[:, :-1] += cn[:, :-1] * phi[:, 1:]
    out[:, 1:] += cn[:, :-1] * phi[:, :-1]
    return out


def boundary_rhs(p, eps, volts, fixed_sides=True):
    """Right-hand side of the boundary potentials (trench_charging_2d.py:323-337)."""
    rhs = np.zeros_like(eps)
    rhs[:, 0] -= 2.0 * eps[:, 0] / p.dx ** 2 * volts["substrate"]
    if p.top_bc == "dirichlet":
        rhs[:, -1] -= 2.0 * eps[:, -1] / p.dx ** 2 * volts["top"]
    top_ox = p.floor_t + p.trench_d
    if p.side_bc == "pillar":
        yfrac = (np.arange(top_ox) + 0.5) / top_ox
        vl = vr = volts["substrate"] + (volts["mask"] - volts["substrate"]) * yfrac
    else:
        vl, vr = (p.left_voltage, p.right_voltage) if fixed_sides else (0.0, 0.0)
    if p.side_bc != "periodic":
        rhs[0, :top_ox] -= 2.0 * eps[0, :top_ox] / p.dx ** 2 * vl
        rhs[-1, :top_ox] -= 2.0 * eps[-1, :top_ox] / p.dx ** 2 * vr
    return rhs


def _grad(c, m, pl, vm, vp, dx):
    """trench_charging_2d.py:429-436"""
    g = np.zeros_like(c)
    g = np.where(vm & vp, (pl - m) / (2 * dx), g)
    g = np.where(vp & ~vm, (pl - c) / dx, g)
    g = np.where(vm & ~vp, (c - m) / dx, g)
    return -g


def compute_field(phi, vac, p, top_voltage=None):
    """E = -grad phi over vacuum neighbours, host version for setup (trench_charging_2d.py:439-454);
    the per-batch field is computed on the device (tb_step_potential)."""
    dx = p.dx
    ex = _grad(phi, np.roll(phi, 1, 0), np.roll(phi, -1, 0), np.roll(vac, 1, 0), np.roll(vac, -1, 0), dx)
    vtop = p.top_voltage if top_voltage is None else top_voltage
    ghost_top = 2 * vtop - phi[:, -1] if p.top_bc == "dirichlet" else phi[:, -1]
    ghost_bot = 2 * p.substrate_voltage - phi[:, 0]
    pd = np.concatenate([ghost_bot[:, None], phi[:, :-1]], axis=1)
    pu = np.concatenate([phi[:, 1:], ghost_top[:, None]], axis=1)
    f = np.zeros((phi.shape[0], 1), dtype=bool)
    vd = np.concatenate([f, vac[:, :-1]], axis=1)
    vu = np.concatenate([vac[:, 1:], ~f], axis=1)
    return ex, _grad(phi, pd, pu, vd, vu, dx)


def circuit_voltages(c, phase):
    """Periodic interpolation of the circuit potentials (trench_charging_2d.py:312-320)."""
    t = np.asarray(c["t"])
    period = (t[1] - t[0]) * t.size
    at = (phase % 360.0) / 360.0 * period
    values = {k: float(np.interp(at, np.append(t, period), np.append(c[k], c[k][0])))
              for k in ("uw", "um", "up", "V1")}
    return dict(substrate=values["uw"] - values["up"], mask=values["um"] - values["up"],
                top=0.0, sheath=values["V1"])


def field_voltages(p, mask, circuit=None):
    """Validation and electrode voltages of setup_fields (trench_charging_2d.py:342-374)."""
    if p.field_mode not in FIELD_MODES or p.side_bc not in SIDE_BCS:
        raise ValueError("invalid field_mode or side_bc")
    if p.top_bc not in ("dirichlet", "neumann"):
        raise ValueError("top_bc must be dirichlet or neumann")
    numeric = (p.rf_phase, p.substrate_voltage, p.mask_voltage, p.top_voltage, p.left_voltage, p.right_voltage)
    if not np.isfinite(numeric).all():
        raise ValueError("voltages and RF phase must be finite")
    driven = p.field_mode != "floating"
    if driven and mask.any() and p.mask_type != "conductor":
        raise ValueError("a mask voltage needs mask_type=conductor")
    if p.side_bc == "pillar" and not driven:
        raise ValueError("the pillar boundary needs field_mode fixed / circuit / circuit_rf")
    if p.field_mode in ("circuit", "circuit_rf"):
        if p.bias != "rf" or circuit is None or p.top_bc != "dirichlet":
            raise ValueError("circuit field modes need bias=rf and top_bc=dirichlet")
    if p.field_mode == "circuit":
        return circuit_voltages(circuit, p.rf_phase)
    if p.field_mode == "circuit_rf":
        if not isinstance(p.rf_time_steps, (int, np.integer)) or p.rf_time_steps < 16:
            raise ValueError("rf_time_steps must be an integer >= 16")
        t = np.asarray(circuit["t"])
        period = (t[1] - t[0]) * t.size
        if (not np.isfinite(period) or period <= 0 or not np.isclose(t[0], 0, atol=period * 1e-12)
                or not np.allclose(np.diff(t), period / t.size, rtol=1e-10, atol=period * 1e-12)):
            raise ValueError("the circuit waveform must be one period sampled evenly from t = 0")
        if not np.isfinite(p.dt_batch) or p.dt_batch < period * (1 - 1e-12):
            raise ValueError("circuit_rf needs dt_batch of at least one RF period")
        wave = np.column_stack((circuit["uw"] - circuit["up"], circuit["um"] - circuit["up"]))
        mean = wave.mean(axis=0)
        return dict(substrate=float(mean[0]), mask=float(mean[1]), top=0.0, sheath=float(np.mean(circuit["V1"])))
    return dict(substrate=p.substrate_voltage, mask=p.mask_voltage, top=p.top_voltage)


class FieldSolver:
    """Multigrid solve of A phi = b on the device with the reference's conductor semantics.

    mode "none": plain solve; "driven": conductor cells held at 0; "floating":
    all conductor cells share one potential set by their total charge (the
    reduced system E^T A E of trench_charging_2d.py:297-309), done here by
    superposition: phi = phi0 + V psi with phi0 solved with the conductor at 0,
    psi the unit-conductor-potential response and V from the conductor row.
    """

    RTOL = 1e-13
    # The FP64 residual b - L x of an n-cell grid cannot be computed below a roundoff floor
    # that grows with the grid (measured: 1.8e-13 relative at 560,000 cells, where 1e-13 is
    # out of reach); the target is RTOL, or 5e-16 sqrt(n) on grids above 40,000 cells.
    # A relative residual of 4e-13 moves the potential by about 1e-7 V.
    RTOL_PER_SQRT_CELL = 5e-16

    def __init__(self, ctx, p, eps, cond, driven, max_rhs=64):
        self.ctx = ctx
        self.nx, self.ny = eps.shape
        self.n = self.nx * self.ny
        self.rtol = max(self.RTOL, self.RTOL_PER_SQRT_CELL * float(np.sqrt(self.n)))
        self.dev = torch.device("cuda", ctx.device)
        self.dx2 = p.dx ** 2
        self.diag, self.ce, self.cn = poisson_matrix_arrays(eps, cond, p)
        self.cond = np.asarray(cond, bool)
        self.mode = "none" if not self.cond.any() else ("driven" if driven else "floating")
        # SPD form L = -dx^2 A
        d = -self.diag * self.dx2
        ke = self.ce * self.dx2
        kn = self.cn * self.dx2
        fixed = self.cond.astype(np.uint8) if self.mode != "none" else np.zeros((self.nx, self.ny), np.uint8)
        self.max_rhs = int(max_rhs)
        self.inner = 12             # FP32 PCG iterations per FP64 refinement step
        self.schedule_used = (1, 1, 16, 12)
        L = _capi.lib()
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        self._operator = (f(d), f(ke), f(kn), np.ascontiguousarray(fixed))
        self._setup(self.max_rhs)
        self.levels = L.tb_poisson_levels(ctx.handle)
        self.cond_t = torch.from_numpy(self.cond.ravel()).to(self.dev)
        self.last_iters = 0
        self.last_resid = 0.0
        if self.mode == "floating":
            # coupling of free cells to the conductor, w_f = sum over conductor neighbours of k_fc
            c = self.cond
            w = np.zeros((self.nx, self.ny))
            east_c, west_c = np.roll(c, -1, axis=0), np.roll(c, 1, axis=0)
            w += np.where(~c & east_c, ke, 0.0)
            w += np.where(~c & west_c, np.roll(ke, 1, axis=0), 0.0)
            w[:, :-1] += np.where(~c[:, :-1] & c[:, 1:], kn[:, :-1], 0.0)
            w[:, 1:] += np.where(~c[:, 1:] & c[:, :-1], kn[:, :-1], 0.0)
            self.w = torch.from_numpy(w.ravel()).to(self.dev)
            psi = self._solve_spd(self.w[None, :].clone())[0]
            self.psi = psi
            self.D = float(d[c].sum()) - float(torch.dot(self.w, psi))

    # device bytes per right-hand side and cell: the solver's FP32/FP64 work vectors on
    # all levels (about 44) plus the FP64 right-hand side, solution and temporaries of
    # solve_rows (about 48)
    BYTES_PER_RHS_CELL = 96

    def _setup(self, max_rhs):
        d, ke, kn, fixed = self._operator
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self.ctx.check(_capi.lib().tb_poisson_setup(self.ctx.handle, ptr(d), ptr(ke), ptr(kn), ptr(fixed),
                                                    int(max_rhs)))
        self.max_rhs = int(max_rhs)

    def resize(self, max_rhs):
        """Right-hand sides per device solve (work vectors are allocated for that many):
        many for the setup's block solves, where each launch of a small grid is latency-
        bound and a wider block needs no more launches, few afterwards to hold less memory."""
        if int(max_rhs) != self.max_rhs:
            self._setup(max_rhs)
            self.set_schedule(*self.schedule_used)

    @classmethod
    def block_size(cls, k, n, budget_bytes=4 << 30):
        """Right-hand sides per block for k solves on n cells within `budget_bytes` of
        device memory."""
        return int(max(1, min(k, budget_bytes // (cls.BYTES_PER_RHS_CELL * n))))

    # work vectors above this size are released after the set-up's block solves
    KEEP_BYTES = 256 << 20

    def _solve_spd(self, bp, x0=None):
        """L x = bp for rows of bp (k, n) on the device (fixed cells must be zero)."""
        L = _capi.lib()
        k = bp.shape[0]
        out = torch.zeros_like(bp) if x0 is None else x0.clone()
        stream = torch.cuda.current_stream(self.dev)
        iters, resid = ctypes.c_int(), ctypes.c_double()
        for s in range(0, k, self.max_rhs):
            e = min(k, s + self.max_rhs)
            b = bp[s:e].contiguous()
            x = out[s:e].contiguous()
            self.ctx.check(L.tb_poisson_solve(self.ctx.handle, e - s, ctypes.c_void_p(b.data_ptr()),
                                              ctypes.c_void_p(x.data_ptr()), self.rtol, 40, self.inner,
                                              ctypes.byref(iters), ctypes.byref(resid),
                                              ctypes.c_void_p(stream.cuda_stream)))
            out[s:e] = x
            self.last_iters = max(self.last_iters, iters.value)
            self.last_resid = max(self.last_resid, resid.value)
        return out

    # candidate V-cycle schedules: (pre, post, coarsest sweeps, PCG iterations per refinement)
    SCHEDULES = ((1, 1, 16, 12), (2, 2, 16, 8), (1, 1, 8, 16), (2, 2, 32, 6), (3, 3, 16, 6))

    def set_schedule(self, pre, post, coarse, inner):
        self.ctx.check(_capi.lib().tb_poisson_schedule(self.ctx.handle, int(pre), int(post), int(coarse)))
        self.inner = int(inner)
        self.schedule_used = (int(pre), int(post), int(coarse), int(inner))

    def autotune(self, b_rows, reps=2):
        """Times the candidate schedules on the right-hand sides b_rows (k, n) (SPD form,
        zero on fixed cells), keeps the fastest and returns {schedule: seconds}."""
        import time
        timings = {}
        for sch in self.SCHEDULES:
            self.set_schedule(*sch)
            best = float("inf")
            for _ in range(reps):
                torch.cuda.synchronize(self.dev)
                t0 = time.perf_counter()
                self._solve_spd(b_rows)
                torch.cuda.synchronize(self.dev)
                best = min(best, time.perf_counter() - t0)
            timings[sch] = best
        self.set_schedule(*min(timings, key=timings.get))
        return timings

    def solve_rows(self, b):
        """A phi = b for the rows of b (k, n) given as a device tensor; returns (k, n)."""
        bp = -self.dx2 * b
        if self.mode == "none":
            return self._solve_spd(bp)
        bc = (bp * self.cond_t).sum(dim=1)                 # conductor part of the right-hand side
        bp = torch.where(self.cond_t[None, :], torch.zeros_like(bp), bp)
        phi0 = self._solve_spd(bp)
        if self.mode == "driven":
            return phi0
        V = (bc + phi0 @ self.w) / self.D
        phi = phi0 + V[:, None] * self.psi[None, :]
        return torch.where(self.cond_t[None, :], V[:, None].expand_as(phi), phi)

    def solve(self, b):
        """Drop-in for fields["solve"]: b is (n,) or (n, k) host or device; returns the same layout."""
        host = not isinstance(b, torch.Tensor)
        bt = torch.as_tensor(np.asarray(b, dtype=np.float64) if host else b, device=self.dev, dtype=torch.float64)
        one = bt.dim() == 1
        rows = bt[None, :] if one else bt.T.contiguous()
        x = self.solve_rows(rows)
        x = x[0] if one else x.T
        return x.cpu().numpy() if host else x


def setup_fields(p, solid, mask, circuit=None, device=0, max_rhs=64):
    """The reference's setup_fields (trench_charging_2d.py:340-413) on the device solver:
    returns dict(solve, cond, eps, external, boundary_rhs, volts, floating, rf, solver),
    with `solve` a FieldSolver.solve (b of A phi = b, flat or column-stacked)."""
    from .tracer import Context
    volts = field_voltages(p, mask, circuit)
    driven = p.field_mode != "floating"
    cond = mask if p.mask_type == "conductor" else np.zeros_like(mask)
    from .geometry import permittivity
    eps = permittivity(solid, mask, p)
    ctx = Context(~solid, device, p.dx)
    solver = FieldSolver(ctx, p, eps, cond, driven, max_rhs=max_rhs)
    nx, ny = solid.shape
    if driven and cond.any():
        phi_cond = cond.astype(float) * volts["mask"]
        mask_rhs = -apply_matrix(solver.diag, solver.ce, solver.cn, phi_cond)
    else:
        phi_cond = np.zeros((nx, ny))
        mask_rhs = np.zeros((nx, ny))
    rhs = boundary_rhs(p, eps, volts)
    external = (solver.solve((rhs + mask_rhs).ravel()) + phi_cond.ravel()).reshape(nx, ny)
    fields = dict(solve=solver.solve, solver=solver, ctx=ctx, cond=cond, eps=eps, external=external,
                  boundary_rhs=rhs, volts=volts, floating=bool(cond.any() and not driven), rf=None)
    if p.field_mode == "circuit_rf":
        t = np.asarray(circuit["t"])
        period = (t[1] - t[0]) * t.size
        wave = np.column_stack((circuit["uw"] - circuit["up"], circuit["um"] - circuit["up"]))
        mean = wave.mean(axis=0)
        basis, rhs_basis = [], []
        for vs, vm in ((1.0, 0.0), (0.0, 1.0)):
            brhs = boundary_rhs(p, eps, dict(substrate=vs, mask=vm, top=0.0), fixed_sides=False)
            bc = cond.astype(float) * vm
            b = brhs - apply_matrix(solver.diag, solver.ce, solver.cn, bc)
            basis.append((solver.solve(b.ravel()) + bc.ravel()).reshape(nx, ny))
            rhs_basis.append(brhs)
        basis = np.array(basis)
        electric = [compute_field(v, ~solid, p, 0.0) for v in basis]
        dt_max = period / p.rf_time_steps
        if p.rf_wave == "pulse":
            dt_max = min(dt_max, p.rf_rise / 8)
        fields["rf"] = dict(period=period, wave=wave - mean, phi=basis, Ex=np.array([e[0] for e in electric]),
                            Ey=np.array([e[1] for e in electric]), dt_max=dt_max, boundary_rhs=np.array(rhs_basis))
    return fields


def conductor_surface_charge(rho, phi, solver, cond, boundary_rhs=None):
    """Charge density for display and saving (trench_charging_2d.py:833-843): rho with the
    conductor cells replaced by the induced surface charge -eps0 (A phi - b) that makes
    them equipotential (during the run a conductor's charge is only a total, kept on one
    cell)."""
    out = np.array(rho, dtype=np.float64, copy=True)
    if np.any(cond):
        induced = apply_matrix(solver.diag, solver.ce, solver.cn, phi)
        if boundary_rhs is not None:
            induced = induced - boundary_rhs
        out[cond] = (-EPS0 * induced)[cond]
    return out


def rf_coefficients(rf, at):
    """Periodic linear interpolation of the voltage deltas (trench_rf.py:5-11)."""
    wave = rf["wave"]
    f = (np.asarray(at) % rf["period"]) / rf["period"] * len(wave)
    i = np.floor(f).astype(np.int64) % len(wave)
    w = (f - np.floor(f))[..., None]
    return wave[i] * (1 - w) + wave[(i + 1) % len(wave)] * w


def field_snapshot(fields, mean_phi, p):
    """Display-phase potential of circuit_rf (trench_charging_2d.py:416-426)."""
    if fields["rf"] is None:
        return mean_phi, fields["external"], fields["boundary_rhs"], fields["volts"]
    rf = fields["rf"]
    delta = rf_coefficients(rf, (p.rf_phase % 360) / 360 * rf["period"])
    shift = np.einsum("i,ijk->jk", delta, rf["phi"])
    rhs = fields["boundary_rhs"] + np.einsum("i,ijk->jk", delta, rf["boundary_rhs"])
    volts = {**fields["volts"], "substrate": fields["volts"]["substrate"] + float(delta[0]),
             "mask": fields["volts"]["mask"] + float(delta[1])}
    return mean_phi + shift, fields["external"] + shift, rhs, volts
