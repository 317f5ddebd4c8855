"""ChargingCase: the reference batch loop with every per-batch stage on the GPU.

Mirrors trench_charging_2d.run (trench_charging_2d.py:1045-1369) for the hot
path: per batch the particles are traced, deposited, leaked, the conductor is
stepped, the potential and field are recomputed and the history is recorded,
all on the device (kernels of libtrench_b200.so) with no host synchronisation.
The host supplies injected particles (``load``), or the caller captures one
batch in a CUDA graph (``capture``) and replays it.

Setup (once per case) builds the multigrid hierarchy, the external potential,
the floating-conductor response, the surface Green's operator G (potential on
the vacuum and surface cells per unit charge density on each surface cell) and
the implicit leakage operator M = inv(I - dt G_leak P) (trench_charging_2d.py:768-803)
from multigrid solves on the GPU.
"""
import ctypes
import json
from dataclasses import asdict, is_dataclass

import numpy as np
import torch

from . import _capi, geometry, steady
from .fields import (FieldSolver, apply_matrix, boundary_rhs, compute_field, conductor_surface_charge,
                     field_snapshot, field_voltages)
from .inject import inject, launch_times
from .params import AMU, E_CHARGE, EPS0, M_E, WALL_MODELS, is_tapered
from .tracer import DEFAULT_VSCALE, Context, _ptr

CLAIM_ORDERS = ("index", "reverse", "learned")     # tb_set_claim_order 0, 1, 2
LEARNED_MIN_CAPACITY = 1 << 16   # default to the learned order from this many particles per batch
HIST_SCALARS = ("ratio_i_bottom", "ratio_e_bottom", "esc_e", "lost", "leak", "particle_steps")
CHECKPOINT_VERSION = 1
# settings a resumed run may change; everything else must equal the saved run's
# (trench_charging_2d.py:951-954; rf_phase too under circuit_rf, where it only moves the display)
RESUME_EDITABLE = frozenset(("until_steady", "n_batches", "max_batches", "steady_window", "steady_rtol",
                             "steady_charge_rtol", "steady_charge_atol", "steady_hold", "backend", "cuda_device",
                             "probe_ions", "probe_energy_eV", "probe_trajectories"))


def validate_resume(res, p):
    """Checks a saved result against the settings of the run that continues it and returns
    the number of batches it holds (the rules of trench_charging_2d.py:959-1007):
    geometry, physics and particle settings unchanged (floats within 1e-9 relative, the
    round trip of a display unit), the same solid and mask, a finite charge of the grid's
    shape, a history with one entry per batch at the batch times, a checkpoint of this
    version holding that many batches and a valid steady streak, and a batch cap beyond
    the saved batches (until_steady) or at least one more batch.  Raises ValueError."""
    params = dict(res.get("params") or {})
    editable = RESUME_EDITABLE | ({"rf_phase"} if params.get("field_mode") == "circuit_rf" else set())
    changed = []
    for k, v in params.items():
        if k in editable or not hasattr(p, k):
            continue
        entered = getattr(p, k)
        same = (bool(np.isclose(entered, v, rtol=1e-9, atol=0)) if isinstance(v, float) and
                isinstance(entered, (int, float)) else entered == v)
        if not same:
            changed.append(k)
    if changed:
        raise ValueError("a resumed run must keep the geometry, physics and particle settings of the saved "
                         "run: " + ", ".join(changed))
    solid, mask, _, _ = geometry.build_geometry(p)
    if ("solid" in res and not np.array_equal(res["solid"], solid)) or (
            "mask" in res and not np.array_equal(res["mask"], mask)):
        raise ValueError("the saved result's geometry differs from this run's")
    rho = np.asarray(res["rho_raw"])
    if rho.shape != solid.shape or not np.isfinite(rho).all():
        raise ValueError("the saved charge has the wrong shape or non-finite values")
    dt = float(params.get("dt_batch", p.dt_batch))
    t = np.asarray((res.get("hist") or {}).get("t", []))
    n = t.size if t.ndim == 1 else 0
    if n == 0 or not np.isfinite(t).all() or not np.allclose(t, np.arange(1, n + 1) * dt, rtol=1e-10,
                                                               atol=dt * 1e-8):
        raise ValueError("resuming needs a continuous history with the batch times")
    for family in ("hist", "charge_hist", "charge_monitor_hist"):
        for name, values in (res.get(family) or {}).items():
            a = np.asarray(values)
            if a.ndim != 1 or len(a) != n or np.isinf(a).any():
                raise ValueError(f"a saved history has the wrong length or infinite values: {family}/{name}")
    ck = res.get("checkpoint")
    if ck and (ck.get("version") != CHECKPOINT_VERSION or ck.get("batches_completed") != n):
        raise ValueError("the saved checkpoint's version or batch count does not match its history")
    hold = int(params.get("steady_hold", p.steady_hold))
    if ck and (not isinstance(ck.get("steady_n_ok"), (int, np.integer)) or not 0 <= ck["steady_n_ok"] <= hold):
        raise ValueError("the saved steady-state streak is invalid")
    if p.until_steady and p.max_batches <= n:
        raise ValueError(f"max_batches counts the whole run: raise it above the {n} saved batches")
    if not p.until_steady and p.n_batches < 1:
        raise ValueError("a resumed run needs at least one more batch")
    return n


class ChargingCase:
    def __init__(self, p, device=0, precision="f32", green="f64", circuit=None, max_batches=None,
                 capacity=None, vscale=DEFAULT_VSCALE, max_rhs=64, autotune=False):
        if precision not in _capi.PRECISION:
            raise ValueError(f"precision must be one of {tuple(_capi.PRECISION)}")
        if green not in ("f32", "f64"):
            raise ValueError("green must be f32 or f64")
        if p.wall_model not in WALL_MODELS:
            raise ValueError(f"wall_model must be one of {WALL_MODELS}: {p.wall_model!r}")
        if not (0 < p.cfl <= 1) or p.max_steps < 1:
            raise ValueError("CUDA tracing needs 0 < cfl <= 1 and max_steps >= 1")
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device is visible (the B200 backend has no CPU path)")
        self.p = p
        self.precision = precision
        self.vscale = float(vscale)
        self.dev = torch.device("cuda", int(device))
        solid, mask, i0, i1 = geometry.build_geometry(p)
        self.solid, self.mask, self.i0, self.i1 = solid, mask, i0, i1
        self.vac = vac = ~solid
        nx, ny = solid.shape
        self.nx, self.ny, self.n = nx, ny, nx * ny
        dev = self.dev
        with torch.cuda.device(dev):
            self.ctx = Context(vac, int(device), p.dx)
            self.volts = volts = field_voltages(p, mask, circuit)
            cond = mask if p.mask_type == "conductor" else np.zeros_like(mask)
            eps = geometry.permittivity(solid, mask, p)
            driven = p.field_mode != "floating"
            self.cond, self.eps = cond, eps
            # the m surface Green's solves run as one block where memory allows (a small grid's
            # solve is launch-bound, so a block of 340 costs about what a block of 64 does); the
            # work vectors are sized for that block from the start
            m_surf = int(geometry.surface_cells(solid).sum())
            wide = max(int(max_rhs), FieldSolver.block_size(m_surf, nx * ny))
            self.solver = solver = FieldSolver(self.ctx, p, eps, cond, driven, max_rhs=wide)
            # external potential (trench_charging_2d.py:378-394)
            if driven and cond.any():
                phi_cond = cond.astype(float) * volts["mask"]
                mask_rhs = -apply_matrix(solver.diag, solver.ce, solver.cn, phi_cond)
            else:
                phi_cond = np.zeros((nx, ny))
                mask_rhs = np.zeros((nx, ny))
            rhs = boundary_rhs(p, eps, volts)
            self.boundary_rhs = rhs
            self.floating = bool(cond.any() and not driven)
            # the external potential's and the floating conductor's solves run in the block of the
            # surface Green's solves below (independent right-hand sides of the same operator)
            extra = [(rhs + mask_rhs).ravel()]
            if self.floating:
                g_rhs = np.zeros(self.n)
                g_rhs[np.flatnonzero(cond)[0]] = -1.0 / (p.dx ** 2 * EPS0)
                extra.append(g_rhs)
            self.driven = driven
            wface = np.where(cond, 1.0, eps / (1.0 + eps))
            self.wface = wface
            # surface cells, Green's rows, probes
            sx, sy = np.nonzero(geometry.surface_cells(solid))
            S = sx * ny + sy
            self.S = S
            m = self.m = len(S)
            self.probes = geometry.probe_cells(solid, p, bool(cond.any()))
            probe_flat = np.array([ix * ny + iy for ix, iy in self.probes.values()], dtype=np.int64)
            rows = np.union1d(np.union1d(np.flatnonzero(vac.ravel()), S), probe_flat)
            self.rows = rows
            self.tuning = {}
            if autotune:
                # the multigrid schedule for the surface Green's solves: timed on a block of them
                k = min(self.solver.max_rhs, m, 64)
                b = torch.zeros((k, self.n), dtype=torch.float64, device=dev)
                b[torch.arange(k, device=dev), torch.from_numpy(S[:k]).to(dev)] = p.dx ** 2 / EPS0
                b = torch.where(self.solver.cond_t[None, :], torch.zeros_like(b), b)
                self.tuning["poisson"] = {str(k_): v for k_, v in self.solver.autotune(b).items()}
            self.tuning["poisson_schedule"] = self.solver.schedule_used
            sol = self._build_green(rows, green, np.array(extra))
            self.external = (sol[0] + phi_cond.ravel()).reshape(nx, ny)
            if solver.max_rhs * self.n * (FieldSolver.BYTES_PER_RHS_CELL // 2) > FieldSolver.KEEP_BYTES:
                solver.resize(max_rhs)
            # leakage (trench_charging_2d.py:768-803)
            self.leak_M = self.leak_h = None
            b0, b1 = geometry.opening_span(solid, p.floor_t)
            e0, e1 = geometry.opening_span(solid, p.floor_t + p.trench_d + p.mask_t - 1)
            self.b0, self.b1, self.e0, self.e1 = b0, b1, e0, e1
            cut = p.floor_t + p.trench_d // 2
            region = geometry.inner_surface_cells(solid, p)[sx, sy] & (sy < cut)
            if p.sigma_s > 0:
                Gl = self._leak_graph(sx, sy)
                self.leak_G = Gl
                P = self.P
                Mt = torch.linalg.inv(torch.eye(m, dtype=torch.float64, device=dev)
                                      - p.dt_batch * (torch.from_numpy(Gl).to(dev) @ P))
                self.leak_M = Mt.contiguous()
                if np.any(self.external):
                    h = p.dt_batch * (Gl @ self.external.ravel()[S])
                    self.leak_h = torch.from_numpy(h).to(dev)
            # floating conductor (trench_charging_2d.py:1087-1090, 807-812)
            self.g_s = None
            self.C_cond, self.c_slot = 0.0, -1
            if self.floating:
                g = sol[1]
                self.g_cond = g.reshape(nx, ny)
                self.C_cond = 1.0 / g[np.flatnonzero(cond)[0]]
                c_cell = np.flatnonzero(geometry.surface_cells(solid) & cond)[0]
                self.c_slot = int(np.flatnonzero(S == c_cell)[0])
                self.g_s = torch.from_numpy(g[S]).to(dev)
            # flags
            sflag = np.zeros(m, np.uint8)
            sflag[cond.ravel()[S]] |= _capi.SFLAG_COND
            sflag[region] |= _capi.SFLAG_REGION
            sflag[(sy == p.floor_t - 1) & (sx >= b0) & (sx < b1)] |= _capi.SFLAG_BOTTOM
            self.q_macro = E_CHARGE * (p.flux * (nx * p.dx) * p.dt_batch / p.n_per_batch)
            # device state
            self.max_batches = int(max_batches or (p.max_batches if p.until_steady else max(p.n_batches, 1)))
            self.hist_cols = len(HIST_SCALARS) + len(self.probes)
            cap = int(capacity or 2 * p.n_per_batch)
            self.capacity = cap
            f64 = torch.float64
            self.t_surf = torch.from_numpy(S.astype(np.int32)).to(dev)
            self.t_sflag = torch.from_numpy(sflag).to(dev)
            self.rho_s = torch.zeros(m, dtype=f64, device=dev)
            self.rho_prev = torch.zeros(m, dtype=f64, device=dev)
            self.work = torch.zeros(2 * m, dtype=f64, device=dev)
            self.t_rows = torch.from_numpy(rows.astype(np.int32)).to(dev)
            self.t_ext = torch.from_numpy(self.external.ravel().copy()).to(dev)
            self.phi = self.t_ext.clone()
            self.ex = torch.zeros(self.n, dtype=f64, device=dev)
            self.ey = torch.zeros(self.n, dtype=f64, device=dev)
            self.t_wface = torch.from_numpy(wface.ravel().copy()).to(dev)
            self.hist = torch.zeros((self.max_batches, self.hist_cols), dtype=f64, device=dev)
            self.t_probes = torch.from_numpy(probe_flat.astype(np.int32)).to(dev)
            self.batch = torch.full((1,), -1, dtype=torch.int32, device=dev)
            self.counts = torch.zeros((2, self.n), dtype=torch.int32, device=dev)
            # charge monitors (trench_charging_2d.py:850-874): weights over the surface slots
            regions = steady.charge_monitors(solid, mask, i0, i1, p)
            self.monitor_names = list(regions) + ["surface absolute"]
            slot = -np.ones(self.n, dtype=np.int64)
            slot[S] = np.arange(m)
            mw = np.zeros((len(self.monitor_names), m))
            for r, cells in enumerate(regions.values()):
                js = slot[cells]
                mw[r, js[js >= 0]] = 1.0
            mw[-1] = mw[list(regions).index("surface")]
            absolute = np.zeros(len(self.monitor_names), np.uint8)
            absolute[-1] = 1
            self.t_mon_w = torch.from_numpy(mw).to(dev)
            self.t_mon_abs = torch.from_numpy(absolute).to(dev)
            self.qhist = torch.zeros((self.max_batches, len(self.monitor_names)), dtype=f64, device=dev)
            self.totals = torch.zeros(8, dtype=torch.int64, device=dev)
            self.X = [torch.zeros(cap, dtype=f64, device=dev) for _ in range(5)]  # x, y, vx, vy, qm
            self.SPC = torch.zeros(cap, dtype=torch.int8, device=dev)
            self._inputs = [(self.X, self.SPC)]   # input buffer sets (a second one for pipelining)
            self.status = torch.full((cap,), 3, dtype=torch.int8, device=dev)
            self.steps = torch.zeros(cap, dtype=torch.int32, device=dev)
            self.n_loaded = 0
            self._desc = self._make_desc(m, sflag)
            self._args = _capi.TraceArgs()
            self._graph = None
            self.trace_events = None   # optional (start, end) CUDA events around the tracer launch
            self.hit = None            # optional (capacity,) int32: absorbing cell of each particle
            self.after_trace = None    # optional callable run on the stream between trace and charge update
            self.rf = None
            if p.field_mode == "circuit_rf":
                self._build_rf(circuit, solver, eps, cond, vac)
            # initial field (trench_charging_2d.py:1198)
            self._potential()
            if self.rf is not None and precision == "f32":
                # the FP32 tracer reads the RF basis in its own packed layout, packed once
                # in the units of the case's field
                wf = _ptr(self.t_wface) if p.wall_model == "barrier" else None
                self.ctx.check(_capi.lib().tb_set_rf_fields(
                    self.ctx.handle, _ptr(self.t_rf["ex"]), _ptr(self.t_rf["ey"]), _ptr(self.t_rf["phi"]), wf,
                    _ptr(self.t_rf["wave"]), len(self.rf["wave"]), self._stream()))
            # FP32 cases of large batches claim in the learned order unless tuned otherwise
            # (adjoint recording of 2^21-particle batches: 10.6 -> 9.0 s); for batches of a few
            # thousand particles the ordering kernels cost more than they save, and circuit_rf
            # launches fall back to index order inside the tracer
            if precision == "f32" and self.rf is None and self.capacity >= LEARNED_MIN_CAPACITY:
                self.set_claim_order(CLAIM_ORDERS.index("learned"))

    # ---- setup helpers -----------------------------------------------------------
    def _build_green(self, rows, green, extra=None):
        """G[r, j] = potential at rows[r] per unit charge density on surface cell j.  `extra`:
        optional (k, n) right-hand sides b of A phi = b solved in the same blocks, ahead of the
        Green's columns; returns their solutions (k, n) on the host."""
        p, dev, S, m = self.p, self.dev, self.S, self.m
        dtype = torch.float32 if green == "f32" else torch.float64
        G = torch.empty((len(rows), m), dtype=dtype, device=dev)
        P = torch.empty((m, m), dtype=torch.float64, device=dev)
        t_rows = torch.from_numpy(rows).to(dev)
        t_S = torch.from_numpy(S).to(dev)
        k_extra = 0 if extra is None else len(extra)
        t_extra = torch.from_numpy(np.ascontiguousarray(extra, dtype=np.float64)).to(dev) if k_extra else None
        solved = []
        chunk = self.solver.max_rhs
        total = k_extra + m
        for s in range(0, total, chunk):
            e = min(total, s + chunk)
            b = torch.zeros((e - s, self.n), dtype=torch.float64, device=dev)
            n_ex = max(0, min(e, k_extra) - s)                 # extra rows in this block
            if n_ex:
                b[:n_ex] = t_extra[s:s + n_ex]
            g0, g1 = s + n_ex - k_extra, e - k_extra            # Green's columns in this block
            if g1 > g0:
                b[n_ex + torch.arange(g1 - g0, device=dev), t_S[g0:g1]] = -1.0 / EPS0
            x = self.solver.solve_rows(b)
            if n_ex:
                solved.append(x[:n_ex].cpu().numpy())
            if g1 > g0:
                G[:, g0:g1] = x[n_ex:, t_rows].T.to(dtype)
                P[:, g0:g1] = x[n_ex:, t_S].T / p.dx ** 2   # per unit charge (1 C/m) on a dx^2 cell
        self.G = G.contiguous()
        self.P = P
        self.green = green
        return np.concatenate(solved) if solved else None

    def _build_rf(self, circuit, solver, eps, cond, vac):
        """Unit-voltage basis of the electrodes and the period-resolved voltage deltas
        (trench_charging_2d.py:397-412); the tracer superposes them in flight."""
        p, dev, nx, ny = self.p, self.dev, self.nx, self.ny
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
        electric = [compute_field(v, vac, p, 0.0) for v in basis]
        dt_max = period / p.rf_time_steps
        if p.rf_wave == "pulse":
            dt_max = min(dt_max, p.rf_rise / 8)
        w = wave - mean
        self.rf = dict(period=float(period), wave=w, phi=basis, Ex=np.array([e[0] for e in electric]),
                       Ey=np.array([e[1] for e in electric]), dt_max=float(dt_max),
                       boundary_rhs=np.array(rhs_basis))
        f = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
        self.t_rf = dict(ex=f(self.rf["Ex"]), ey=f(self.rf["Ey"]), phi=f(basis), wave=f(w))
        bound = np.abs(w).max(axis=0)
        self.rf_bound = (float(bound[0]), float(bound[1]))
        self.clock = torch.zeros((self.capacity, 2), dtype=torch.float64, device=dev)

    def _leak_graph(self, sx, sy):
        """Conductance graph of the surface cells (trench_charging_2d.py:778-792)."""
        p, nx, ny, m = self.p, self.nx, self.ny, self.m
        smap = -np.ones((nx, ny), dtype=np.int64)
        smap[sx, sy] = np.arange(m)
        g = p.sigma_s / p.dx
        G = np.zeros((m, m))
        for a, b in ((smap, np.roll(smap, -1, axis=0)), (smap[:, :-1], smap[:, 1:])):
            sel = (a >= 0) & (b >= 0)
            a, b = a[sel], b[sel]
            np.add.at(G, (a, b), g)
            np.add.at(G, (b, a), g)
            np.add.at(G, (a, a), -g)
            np.add.at(G, (b, b), -g)
        return G

    def _make_desc(self, m, sflag):
        p = self.p
        d = _capi.StepDesc()
        d.m = m
        d.d_surf, d.d_sflag = _ptr(self.t_surf), _ptr(self.t_sflag)
        d.d_rho_s, d.d_rho_prev, d.d_work = _ptr(self.rho_s), _ptr(self.rho_prev), _ptr(self.work)
        d.d_leak_M, d.d_leak_h, d.d_g_s = _ptr(self.leak_M), _ptr(self.leak_h), _ptr(self.g_s)
        d.c_slot = self.c_slot
        d.floating, d.driven = int(self.floating), int(self.driven)
        d.q_macro, d.dx, d.C_cond, d.Te = self.q_macro, float(p.dx), float(self.C_cond), float(p.electron_temp_eV)
        d.dt_batch = float(p.dt_batch)
        d.leak_norm = float(E_CHARGE * p.flux * (self.e1 - self.e0) * p.dx)
        d.bottom_norm = float(p.n_per_batch * ((self.b1 - self.b0) / self.nx))
        d.n_per_batch = float(p.n_per_batch)
        d.n_rows = len(self.rows)
        d.d_rows = _ptr(self.t_rows)
        d.d_green = _ptr(self.G) if self.green == "f32" else None
        d.d_green64 = _ptr(self.G) if self.green == "f64" else None
        d.d_ext, d.d_phi = _ptr(self.t_ext), _ptr(self.phi)
        d.d_ex, d.d_ey = _ptr(self.ex), _ptr(self.ey)
        d.d_wface = _ptr(self.t_wface) if p.wall_model == "barrier" else None
        d.v_sub, d.v_top = float(p.substrate_voltage), float(self.volts["top"])
        d.top_dirichlet = int(p.top_bc == "dirichlet")
        d.vscale = self.vscale
        d.d_hist = _ptr(self.hist)
        d.hist_cols, d.max_batches = self.hist_cols, self.max_batches
        d.n_probes = len(self.probes)
        d.d_probes, d.d_batch = _ptr(self.t_probes), _ptr(self.batch)
        d.d_counts, d.d_totals = _ptr(self.counts), _ptr(self.totals)
        return d

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def _potential(self):
        self.ctx.check(_capi.lib().tb_step_potential(self.ctx.handle, ctypes.byref(self._desc), self._stream()))

    # ---- per batch -----------------------------------------------------------------
    def load(self, x, y, vx, vy, qm, spc, non_blocking=False, launch_times=None):
        """Copy one batch of injected particles into the device buffers (with their RF
        launch times in circuit_rf mode)."""
        n = len(x)
        if self.rf is not None:
            if launch_times is None or len(launch_times) != n:
                raise ValueError("circuit_rf needs one launch time per particle")
            t0 = np.asarray(launch_times, dtype=np.float64) % self.rf["period"]
            self.clock[:n].copy_(torch.from_numpy(np.column_stack((t0, np.zeros(n)))), non_blocking=False)
        if n > self.capacity:
            raise ValueError(f"{n} particles exceed the case capacity {self.capacity}")
        if any(len(v) != n for v in (y, vx, vy, qm, spc)):
            raise ValueError("particle arrays differ in length")
        for dst, src in zip(self.X, (x, y, vx, vy, qm)):
            t = src if isinstance(src, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(src, np.float64))
            dst[:n].copy_(t, non_blocking=non_blocking)
        t = spc if isinstance(spc, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(spc, np.int8))
        self.SPC[:n].copy_(t, non_blocking=non_blocking)
        self.n_loaded = n

    def _load_staged(self, parts, launch_times=None):
        """load() for host arrays without waiting for the device: the batch goes into one of
        two pinned staging buffers and is copied on the stream behind the previous batch's
        work, so the host draws batch k+1 while the device runs batch k.  A staging buffer
        is written again only after its previous copy has run (its event)."""
        n = len(parts[0])
        if n > self.capacity:
            raise ValueError(f"{n} particles exceed the case capacity {self.capacity}")
        if any(len(v) != n for v in parts[1:]):
            raise ValueError("particle arrays differ in length")
        if self.rf is not None and (launch_times is None or len(launch_times) != n):
            raise ValueError("circuit_rf needs one launch time per particle")
        if not hasattr(self, "_staging"):
            cap = self.capacity
            self._staging = [[torch.empty(cap, dtype=torch.float64).pin_memory() for _ in range(5)]
                             + [torch.empty(cap, dtype=torch.int8).pin_memory(),
                                torch.empty((cap, 2), dtype=torch.float64).pin_memory()] for _ in range(2)]
            self._staging_done = [None, None]
            self._staging_k = 0
        j = self._staging_k % 2
        self._staging_k += 1
        if self._staging_done[j] is not None:
            self._staging_done[j].synchronize()
        buf = self._staging[j]
        for dst, src in zip(buf[:5], parts[:5]):
            np.copyto(dst[:n].numpy(), src, casting="same_kind")
        np.copyto(buf[5][:n].numpy(), parts[5], casting="unsafe")
        for dst, src in zip(self.X + [self.SPC], buf[:6]):
            dst[:n].copy_(src[:n], non_blocking=True)
        if self.rf is not None:
            clk = buf[6][:n].numpy()
            clk[:, 0] = np.asarray(launch_times, dtype=np.float64) % self.rf["period"]
            clk[:, 1] = 0.0
            self.clock[:n].copy_(buf[6][:n], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.dev))
        self._staging_done[j] = ev
        self.n_loaded = n

    def add_input_buffer(self):
        """A second set of particle input buffers, so the next batch can be copied in while
        the current one runs (see HostPipeline)."""
        if len(self._inputs) < 2:
            X = [torch.zeros(self.capacity, dtype=torch.float64, device=self.dev) for _ in range(5)]
            self._inputs.append((X, torch.zeros(self.capacity, dtype=torch.int8, device=self.dev)))
        return self._inputs[1]

    def _fill_args(self, n, buffer=0):
        """Tracer arguments of one batch of n particles in input buffer set `buffer`;
        returns the precision of the kernel that traces it."""
        p = self.p
        X, SPC = self._inputs[buffer]
        a = self._args
        a.n = n
        a.d_x, a.d_y, a.d_vx, a.d_vy, a.d_qm = (_ptr(t) for t in X)
        a.d_spc = _ptr(SPC)
        a.d_ex, a.d_ey = _ptr(self.ex), _ptr(self.ey)
        bar = p.wall_model == "barrier"
        a.d_phi, a.d_wface = (_ptr(self.phi), _ptr(self.t_wface)) if bar else (None, None)
        a.max_steps = a.step_budget = int(p.max_steps)
        a.cfl = float(p.cfl)
        a.tapered = int(is_tapered(p))
        a.d_counts, a.d_totals = _ptr(self.counts), _ptr(self.totals)
        a.d_status, a.d_steps = _ptr(self.status), _ptr(self.steps)
        a.d_hit = _ptr(self.hit) if self.hit is not None else None
        a.write_state = 0
        precision = self.precision
        if self.rf is not None:
            # the in-flight RF clock (precision f32 reads the basis packed at set-up)
            a.d_rf_ex, a.d_rf_ey, a.d_rf_phi = _ptr(self.t_rf["ex"]), _ptr(self.t_rf["ey"]), _ptr(self.t_rf["phi"])
            a.d_wave = _ptr(self.t_rf["wave"])
            a.n_phase = len(self.rf["wave"])
            a.period, a.dt_max = self.rf["period"], self.rf["dt_max"]
            a.bound_vs, a.bound_vm = self.rf_bound
            a.d_clock = _ptr(self.clock)
        return precision

    def step(self, n=None, buffer=0):
        """One charging batch on the current stream (trace, deposit, leakage, conductor, potential, field),
        reading the particles from input buffer set `buffer`."""
        L = _capi.lib()
        n = self.n_loaded if n is None else n
        s = self._stream()
        self.ctx.check(L.tb_batch_reset(self.ctx.handle, _ptr(self.status), _ptr(self.steps), n, _ptr(self.counts),
                                        self.counts.numel(), _ptr(self.totals), self.totals.numel(), s))
        a = self._args
        precision = self._fill_args(n, buffer)
        ev = getattr(self, "trace_events", None)
        if ev is not None:
            ev[0].record()
        if n:
            self.ctx.check(L.tb_trace(self.ctx.handle, ctypes.byref(a), _capi.PRECISION[precision], s))
        if ev is not None:
            ev[1].record()
        if self.after_trace is not None:
            self.after_trace()
        self.ctx.check(L.tb_step_charge(self.ctx.handle, ctypes.byref(self._desc), s))
        # the charge monitors read only the new charge and the batch row: they run on a
        # second stream beside the potential and field update (a fork and join inside a
        # captured graph)
        cur = torch.cuda.current_stream(self.dev)
        if not hasattr(self, "_side"):
            self._side = torch.cuda.Stream(self.dev)
            self._ev_fork, self._ev_join = torch.cuda.Event(), torch.cuda.Event()
        self._ev_fork.record(cur)
        self._side.wait_event(self._ev_fork)
        self.ctx.check(L.tb_step_monitors(self.ctx.handle, ctypes.byref(self._desc), _ptr(self.t_mon_w),
                                          _ptr(self.t_mon_abs), len(self.monitor_names), _ptr(self.qhist),
                                          ctypes.c_void_p(self._side.cuda_stream)))
        self._ev_join.record(self._side)
        self.ctx.check(L.tb_step_potential(self.ctx.handle, ctypes.byref(self._desc), s))
        cur.wait_event(self._ev_join)

    TRACER_SHAPES = ((1024, 1), (768, 1), (512, 1), (512, 2), (256, 1), (128, 1))

    def set_claim_order(self, order):
        """Sets the tracer's claim order (an index into CLAIM_ORDERS); the learned order's
        buffers are reserved for the case's capacity, so graphs captured later use it."""
        L = _capi.lib()
        self.ctx.check(L.tb_set_claim_order(self.ctx.handle, int(order)))
        if CLAIM_ORDERS[order] == "learned":
            self.ctx.check(L.tb_reserve_claim_order(self.ctx.handle, self.capacity))
        self.tuning["claim_order"] = CLAIM_ORDERS[order]

    def autotune_tracer(self, n=None, reps=2):
        """Times the tracer's launch shapes (CTA size, CTAs per SM) and claim orders (index
        order, from the last index down, or learned: electrons first, then ions longest
        predicted first) on the loaded batch and keeps the fastest.
        Traces only: neither the charge state nor the loaded batch is changed (the trace
        is deterministic, so every setting gives the same counts)."""
        L = _capi.lib()
        n = self.n_loaded if n is None else n
        timings = {}
        saved = self.trace_events
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        self.trace_events = (e0, e1)
        try:
            for order in range(len(CLAIM_ORDERS)):
                self.set_claim_order(order)
                for threads, per_sm in self.TRACER_SHAPES:
                    self.ctx.check(L.tb_set_tuning(self.ctx.handle, threads, per_sm))
                    best = float("inf")
                    for _ in range(reps):
                        self._trace_only(n)
                        e1.synchronize()
                        best = min(best, e0.elapsed_time(e1))
                    timings[(threads, per_sm, order)] = best
        finally:
            self.trace_events = saved
        threads, per_sm, order = min(timings, key=timings.get)
        self.ctx.check(L.tb_set_tuning(self.ctx.handle, threads, per_sm))
        self.set_claim_order(order)
        self.tuning["tracer"] = {f"{t}x{c}{'-' + CLAIM_ORDERS[o] if o else ''}": v for (t, c, o), v in timings.items()}
        self.tuning["tracer_shape"] = (threads, per_sm)
        self.tuning["claim_order"] = CLAIM_ORDERS[order]
        return timings

    def _trace_only(self, n):
        """The tracer launch of step() alone (counts and status are overwritten by the next step).
        The tracer writes the state of particles still live at the step cap back to its
        inputs, so the launch traces a copy of the loaded batch (in the second input
        buffer set) and leaves the batch itself as it was."""
        L = _capi.lib()
        s = self._stream()
        X1, S1 = self.add_input_buffer()
        for dst, src in zip(X1 + [S1], self.X + [self.SPC]):
            dst[:n].copy_(src[:n])
        self.status[:n].fill_(3)
        self.steps[:n].zero_()
        self.counts.zero_()
        self.totals.zero_()
        precision = self._fill_args(n, 1)
        clock = self.clock[:n].clone() if self.rf is not None else None   # in/out RF launch clocks
        ev = self.trace_events
        if ev is not None:
            ev[0].record()
        self.ctx.check(L.tb_trace(self.ctx.handle, ctypes.byref(self._args), _capi.PRECISION[precision], s))
        if ev is not None:
            ev[1].record()
        if clock is not None:
            self.clock[:n].copy_(clock)

    def capture(self, n=None, buffer=0):
        """Capture one batch (for n particles in input buffer set `buffer`) as a CUDA graph."""
        n = self.n_loaded if n is None else n
        side = torch.cuda.Stream(self.dev)
        side.wait_stream(torch.cuda.current_stream(self.dev))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            with torch.cuda.graph(g, stream=side):
                self.step(n, buffer)
        torch.cuda.current_stream(self.dev).wait_stream(side)
        if buffer == 0:
            self._graph = g
        return g

    def replay(self):
        self._graph.replay()

    def check(self):
        """Synchronise and raise if a kernel recorded a failed check."""
        self.ctx.check(_capi.lib().tb_check(self.ctx.handle, self._stream()))

    # ---- results -------------------------------------------------------------------
    def batches_done(self):
        return int(self.batch.item()) + 1

    def history(self):
        nb = min(self.batches_done(), self.max_batches)
        h = self.hist[:nb].cpu().numpy()
        out = {k: h[:, i].copy() for i, k in enumerate(HIST_SCALARS)}
        for j, k in enumerate(self.probes):
            out[k] = h[:, len(HIST_SCALARS) + j].copy()
        out["t"] = np.arange(1, nb + 1) * self.p.dt_batch
        return out

    def charge_history(self):
        """Charge monitors per batch (C/m): the reference's charge_monitor_hist; its
        charge_hist is the 'left' and 'right' entries."""
        nb = min(self.batches_done(), self.max_batches)
        q = self.qhist[:nb].cpu().numpy()
        return {k: q[:, r].copy() for r, k in enumerate(self.monitor_names)}

    def rho(self):
        r = np.zeros(self.n)
        r[self.S] = self.rho_s.cpu().numpy()
        return r.reshape(self.nx, self.ny)

    def compare_precisions(self, batch):
        """The FP32 tracer against the FP64 one on one batch from the case's current state:
        the same particles (host arrays x, y, vx, vy, qm, spc) traced by both kernels from
        the same charge, each followed by the same charge update; the case is left as it
        was.  Returns the per-particle agreement of status and absorbing cell, the bottom
        ion-flux ratio of the batch under each (difference in % and in units of its
        counting noise) and the largest potential difference after the update over every
        cell (V)."""
        ck = self.checkpoint()
        n = len(batch[0])
        saved_hit, saved_precision = self.hit, self.precision
        self.hit = torch.full((self.capacity,), -1, dtype=torch.int32, device=self.dev)
        out = {}
        try:
            for prec in ("f32", "f64"):
                self.restore(ck)
                self.precision = prec
                self.hit.fill_(-1)
                self.load(*batch)
                self.step(n)
                torch.cuda.synchronize(self.dev)
                out[prec] = dict(status=self.status[:n].cpu().numpy(), hit=self.hit[:n].cpu().numpy(),
                                 ratio=float(self.history()["ratio_i_bottom"][-1]), phi=self.full_potential())
        finally:
            self.precision = saved_precision
            self.hit = saved_hit
            self.restore(ck)
        a, b = out["f32"], out["f64"]
        same = (a["status"] == b["status"]) & (a["hit"] == b["hit"])
        norm = self.p.n_per_batch * (self.b1 - self.b0) / self.nx
        sigma = np.sqrt(max(b["ratio"] * norm, 1.0)) / norm
        return {"particles": n, "hit_agreement": float(same.mean()), "differing": int((~same).sum()),
                "ratio_i_bottom": {"f32": a["ratio"], "f64": b["ratio"],
                                   "error_pct": 100.0 * abs(a["ratio"] - b["ratio"]) / max(abs(b["ratio"]), 1e-300),
                                   "error_sigma": abs(a["ratio"] - b["ratio"]) / sigma},
                "potential_max_abs_diff_V": float(np.abs(a["phi"] - b["phi"]).max())}

    def full_potential(self):
        """phi on every cell: solve(-rho/eps0) + external (trench_charging_2d.py:1268)."""
        rho = self.rho()
        return (self.solver.solve((-rho / EPS0).ravel()) + self.external.ravel()).reshape(self.nx, self.ny)

    def fields(self):
        return (self.ex.cpu().numpy().reshape(self.nx, self.ny), self.ey.cpu().numpy().reshape(self.nx, self.ny))

    # ---- checkpoint / resume ---------------------------------------------------------
    def checkpoint(self, rng=None, phase_rng=None):
        """State to continue from: the surface charge (as the reference's full-grid rho_raw),
        the history and the generator states (trench_charging_2d.py:1361-1364).  Everything
        else on the device is recomputed from the charge."""
        self.check()
        params = asdict(self.p) if is_dataclass(self.p) else dict(vars(self.p))
        return dict(rho_raw=self.rho(), hist=self.history(), params=params,
                    charge_monitor_hist=self.charge_history(),
                    checkpoint=dict(version=CHECKPOINT_VERSION, batches_completed=self.batches_done(),
                                    rng_state=rng.bit_generator.state if rng is not None else None,
                                    phase_rng_state=phase_rng.bit_generator.state if phase_rng is not None
                                    else None,
                                    steady_n_ok=int(getattr(self, "_steady_n_ok", 0))))

    def restore(self, res):
        """Continue from a checkpoint of this backend or a reference result of the same case
        (keys rho_raw, hist): charge, history rows and batch counter."""
        rho = np.asarray(res["rho_raw"], dtype=np.float64)
        if rho.shape != (self.nx, self.ny) or not np.isfinite(rho).all():
            raise ValueError("the checkpoint's charge does not match this geometry")
        off = np.ones(self.n, bool)
        off[self.S] = False
        if np.any(rho.ravel()[off] != 0):
            raise ValueError("the checkpoint holds charge outside the surface cells")
        hist = res.get("hist", {})
        t = np.asarray(hist.get("t", []))
        done = len(t)
        if done > self.max_batches:
            raise ValueError("the checkpoint has more batches than this case's history holds")
        rows = np.zeros((done, self.hist_cols))
        for i, k in enumerate(HIST_SCALARS):
            if k in hist:
                rows[:, i] = np.asarray(hist[k], dtype=np.float64)[:done]
        for j, k in enumerate(self.probes):
            if k in hist:
                rows[:, len(HIST_SCALARS) + j] = np.asarray(hist[k], dtype=np.float64)[:done]
        # charge monitors: the saved ones, NaN where the result has none (the steady-state
        # check then starts after them, as the reference's steady_history_start does)
        mon = res.get("charge_monitor_hist", {}) or {}
        qrows = np.full((done, len(self.monitor_names)), np.nan)
        for r, k in enumerate(self.monitor_names):
            if k in mon and len(mon[k]) >= done:
                qrows[:, r] = np.asarray(mon[k], dtype=np.float64)[:done]
        with torch.cuda.device(self.dev):
            self.rho_s.copy_(torch.from_numpy(rho.ravel()[self.S].copy()))
            self.hist.zero_()
            self.qhist.zero_()
            if done:
                self.hist[:done].copy_(torch.from_numpy(rows))
                self.qhist[:done].copy_(torch.from_numpy(qrows))
            self.batch.fill_(done - 1)
            self._potential()
            torch.cuda.current_stream(self.dev).synchronize()

    def save(self, path, rng=None, phase_rng=None):
        """NPZ without pickled objects: arrays plus JSON text (like trench_charging_2d.py:1720-1733)."""
        ck = self.checkpoint(rng, phase_rng)
        np.savez(path, rho_raw=ck["rho_raw"], params_json=json.dumps(ck["params"]),
                 checkpoint_json=json.dumps(ck["checkpoint"]),
                 monitor_names_json=json.dumps(list(ck["charge_monitor_hist"])),
                 monitors=np.array(list(ck["charge_monitor_hist"].values())),
                 **{f"hist_{k}": v for k, v in ck["hist"].items()})

    @staticmethod
    def load_checkpoint(path):
        """Read a file written by save()."""
        with np.load(path, allow_pickle=False) as d:
            res = dict(rho_raw=d["rho_raw"], params=json.loads(str(d["params_json"])),
                       checkpoint=json.loads(str(d["checkpoint_json"])),
                       hist={k[5:]: d[k] for k in d.files if k.startswith("hist_")})
            if "monitor_names_json" in d.files:
                res["charge_monitor_hist"] = dict(zip(json.loads(str(d["monitor_names_json"])), d["monitors"]))
        return res

    @staticmethod
    def restore_rng(state):
        """A numpy Generator positioned at a saved PCG64 state (trench_charging_2d.py:1012-1031)."""
        rng = np.random.default_rng()
        rng.bit_generator.state = state
        return rng

    STEADY_SETTINGS = ("until_steady", "steady_window", "steady_rtol", "steady_charge_rtol",
                       "steady_charge_atol", "steady_hold")

    def run(self, n_batches=None, rng=None, ion_energy=None, ion_velocity=None, log=None, resume=None, stop=None,
            injector=None):
        """The reference batch loop (trench_charging_2d.py:1199-1369) with host injection,
        or with `injector` (an inject.DeviceInjector of this case) drawing every batch on
        the device, each batch then replayed from one CUDA graph (inject + step).
        Without until_steady it runs n_batches (default p.n_batches) more batches; with
        until_steady it runs until the steady-state check (potential probes and charge
        monitors, every steady_window batches) has passed steady_hold times in a row or
        p.max_batches batches are done.  `resume` (a checkpoint or loaded file, or a
        reference result) continues a saved run; `stop` (an object with is_set()) ends
        the loop between batches."""
        p = self.p
        phase_rng = None
        n_ok = 0
        if resume is not None:
            validate_resume(resume, p)
            self.restore(resume)
            ck = resume.get("checkpoint") or {}
            if rng is None and ck.get("rng_state"):
                rng = self.restore_rng(ck["rng_state"])
            if self.rf is not None and ck.get("phase_rng_state"):
                phase_rng = self.restore_rng(ck["phase_rng_state"])
            src = resume.get("params") or {}
            if p.until_steady and ck.get("steady_n_ok") is not None and all(
                    src.get(k) == getattr(p, k) for k in self.STEADY_SETTINGS):
                n_ok = int(ck["steady_n_ok"])
        rng = np.random.default_rng(p.seed) if rng is None else rng
        if p.field_mode in ("circuit", "circuit_rf") and ion_energy is None and ion_velocity is None:
            # ions start at the plasma potential with the Bohm energy (trench_charging_2d.py:1135-1139)
            ion_energy = lambda r, k: np.full(k, p.electron_temp_eV / 2)
        if phase_rng is None and self.rf is not None:
            phase_rng = np.random.default_rng(np.random.SeedSequence([p.seed, 0x5246]))
        self._rngs = (rng, phase_rng)
        start = self.batches_done()
        if p.until_steady:
            n_max = int(p.max_batches)
        else:
            n_max = start + int(p.n_batches if n_batches is None else n_batches)
        if n_max > self.max_batches:
            raise ValueError(f"{n_max} batches exceed this case's history of {self.max_batches} "
                             "(ChargingCase(max_batches=...))")
        W = int(p.steady_window)
        probes = list(self.probes)
        # potentials are compared with the external ones only under the RF circuit
        # (trench_charging_2d.py:1167-1168)
        reference = ({k: float(self.external[ix, iy]) for k, (ix, iy) in self.probes.items()}
                     if self.rf is not None else None)
        first = 0
        if p.until_steady and start:
            first = steady.history_start(self.history(), probes, self.charge_history())
        converged_at, stopped, check = None, False, None
        graph = None
        with torch.cuda.device(self.dev):
            for b in range(start, n_max):
                if stop is not None and stop.is_set():
                    stopped = True
                    break
                if injector is not None:
                    if graph is None and b > start:
                        # inject + step as one graph; the injector's Philox batch word follows the
                        # case's device batch counter, so every replay draws a new batch
                        side = torch.cuda.Stream(self.dev)
                        side.wait_stream(torch.cuda.current_stream(self.dev))
                        graph = torch.cuda.CUDAGraph()
                        with torch.cuda.stream(side), torch.cuda.graph(graph, stream=side):
                            injector()
                            self.step(2 * p.n_per_batch)
                        torch.cuda.current_stream(self.dev).wait_stream(side)
                    if graph is not None:
                        graph.replay()
                    else:
                        injector()
                        self.step()
                else:
                    parts = inject(p, p.n_per_batch, self.ny, rng, ion_energy, ion_velocity)
                    t0 = None
                    if phase_rng is not None:
                        t0 = np.concatenate([launch_times(phase_rng, p.n_per_batch, self.rf["period"])
                                             for _ in range(2)])
                    self._load_staged(parts, launch_times=t0)
                    self.step()
                if log is not None and ((b + 1) % 10 == 0 or b == 0):
                    log(f"[{b + 1}/{n_max}]")
                if p.until_steady and (b + 1) % W == 0 and (b + 1) - first >= 2 * W:
                    hist, mon = self.history(), self.charge_history()
                    v_ok, name, d, tol = steady.check_steady(hist, probes, p, reference)
                    charge = steady.check_charge_steady(mon, p)
                    ok = bool(v_ok and charge["ok"])
                    n_ok = min(n_ok + 1, p.steady_hold) if ok else 0
                    check = dict(ok=ok, n_ok=n_ok, voltage=dict(ok=bool(v_ok), name=name, d=float(d), tol=float(tol)),
                                 charge=charge)
                    if log is not None:
                        log(f"  steady check: potential {'OK' if v_ok else 'NG'} ({name} {d:+.3g} V, tol {tol:.3g}), "
                            f"charge {'OK' if charge['ok'] else 'NG'} ({charge['name']} {charge['kind']}) "
                            f"-> {n_ok}/{p.steady_hold}")
                    if n_ok >= p.steady_hold:
                        converged_at = b + 1
                        break
            del graph
            self.check()
        self._steady_n_ok = n_ok
        ex, ey = self.fields()
        mean_phi = self.full_potential()
        rho_raw = self.rho()
        # display phase of circuit_rf (trench_charging_2d.py:416-426, 1355-1359)
        shown_phi, external, shown_rhs, volts = field_snapshot(
            dict(rf=self.rf, external=self.external, boundary_rhs=self.boundary_rhs, volts=self.volts), mean_phi, p)
        if self.rf is not None:
            ex, ey = compute_field(shown_phi, self.vac, p, volts["top"])
        hist = self.history()
        ck = self.checkpoint(rng, phase_rng)["checkpoint"]
        mon = self.charge_history()
        Wl = min(W, len(hist["t"]))
        steady_values = {k: float(hist[k][-Wl:].mean()) for k in probes} if Wl else {}
        t_conv = converged_at * p.dt_batch if converged_at else np.nan
        if p.until_steady and log is not None and not converged_at and not stopped:
            log(f"not steady after {n_max} batches (raise max_batches)")
        params = asdict(p) if is_dataclass(p) else dict(vars(p))
        return dict(phi=shown_phi, mean_phi=mean_phi,
                    rho=conductor_surface_charge(rho_raw, shown_phi, self.solver, self.cond, shown_rhs),
                    Ex=ex, Ey=ey, rho_raw=rho_raw, external_phi=external, voltages=volts, hist=hist,
                    charge_hist={k: mon[k] for k in ("left", "right")}, charge_monitor_hist=mon,
                    steady=steady_values, t_conv=t_conv, converged=converged_at is not None, stopped=stopped,
                    check=check, start_batch=start, params=params,
                    solid=self.solid, mask=self.mask, probes=self.probes, backend_used="b200", checkpoint=ck)


class HostPipeline:
    """Batches from pinned host memory with the copy of batch k+1 overlapping the
    compute of batch k: two input buffer sets, one CUDA graph per set, a copy stream.
    The reference's loop (trench_charging_2d.py:1225-1285) copies and computes one
    batch after the other.

    A batch is (x, y, vx, vy, qm, spc) like the reference's, or (x, y, vx, vy, spc): then
    each particle's charge-to-mass ratio is its species' (ions e / (ion_mass_amu u),
    electrons -e / m_e, as the reference's inject draws them, trench_charging_2d.py:
    458-489) and is written on the device from the species, so the host link carries
    33 of the 41 bytes per particle (the link, about 22 GB/s from pinned memory on the
    B200 hosts measured, is slower than the tracer at 41 bytes)."""

    def __init__(self, case, n):
        self.case = case
        self.n = int(n)
        case.add_input_buffer()
        self.graphs = [case.capture(self.n, 0), case.capture(self.n, 1)]
        self.copy = torch.cuda.Stream(case.dev)
        self.copied = [torch.cuda.Event(), torch.cuda.Event()]
        self.done = [torch.cuda.Event(), torch.cuda.Event()]
        self.row_dev = [torch.empty(case.hist_cols, dtype=torch.float64, device=case.dev) for _ in range(2)]
        qm_ion = E_CHARGE / (case.p.ion_mass_amu * AMU)
        self.qm_species = (torch.tensor(qm_ion, dtype=torch.float64, device=case.dev),
                           torch.tensor(-E_CHARGE / M_E, dtype=torch.float64, device=case.dev))

    def _stage(self, k, batch, after):
        X, SPC = self.case._inputs[k % 2]
        if len(batch) not in (5, 6):
            raise ValueError("a batch is (x, y, vx, vy, qm, spc) or (x, y, vx, vy, spc)")
        self.copy.wait_event(after)
        with torch.cuda.stream(self.copy):
            if len(batch) == 6:
                for dst, src in zip(X + [SPC], batch):
                    dst[:self.n].copy_(src, non_blocking=True)
            else:
                for dst, src in zip(X[:4] + [SPC], batch):
                    dst[:self.n].copy_(src, non_blocking=True)
                torch.where(SPC[:self.n] == 0, self.qm_species[0], self.qm_species[1], out=X[4][:self.n])
            self.copied[k % 2].record(self.copy)

    def run(self, batches, rows=None, between=None):
        """batches: list of pinned host tensors of n particles each, (x, y, vx, vy, qm, spc)
        or (x, y, vx, vy, spc) with the species' charge-to-mass ratios.
        rows: optional pinned (len(batches), hist_cols) tensor receiving each batch's
        history row.  between: optional callable run on the compute stream between batches."""
        comp = torch.cuda.current_stream(self.case.dev)
        start = torch.cuda.Event()
        start.record(comp)
        self._stage(0, batches[0], start)
        for k in range(len(batches)):
            comp.wait_event(self.copied[k % 2])
            if k + 1 < len(batches):
                # buffer (k+1)%2 is free once batch k-1 has finished with it
                self._stage(k + 1, batches[k + 1], self.done[(k + 1) % 2] if k >= 1 else start)
            self.graphs[k % 2].replay()
            if rows is not None:
                # the history row is gathered on the compute stream and read back on the copy
                # stream, so the device-to-host transfer stays off the compute path
                last = self.case.batch.clamp(0, self.case.max_batches - 1).long()
                self.row_dev[k % 2].copy_(self.case.hist.index_select(0, last).squeeze(0))
            self.done[k % 2].record(comp)
            if rows is not None:
                self.copy.wait_event(self.done[k % 2])
                with torch.cuda.stream(self.copy):
                    rows[k].copy_(self.row_dev[k % 2], non_blocking=True)
            if between is not None:
                between()
        comp.wait_stream(self.copy)   # the last history rows are on the host when the stream is done
