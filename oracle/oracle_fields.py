"""ORACLE -- test infrastructure only (the checker, never the product).

NumPy/SciPy restatement of the field side of the reference charging step and of
its batch loop, used to check the CUDA path:

  poisson_matrix      trench_charging_2d.py:252-294   (5-point FV, harmonic face eps)
  make_solver         trench_charging_2d.py:297-309   (SuperLU, floating conductor collapsed)
  boundary_rhs        trench_charging_2d.py:323-337
  setup_fields        trench_charging_2d.py:340-413   (floating / fixed / circuit_rf basis)
  compute_field       trench_charging_2d.py:429-454
  surface_cells       trench_charging_2d.py:734-752
  build_leakage       trench_charging_2d.py:768-803
  conductor_response  trench_charging_2d.py:807-812
  conductor_step      trench_charging_2d.py:815-830
  batch_update        trench_charging_2d.py:1239-1285 (one batch after the trace)

Geometry (solid, mask) is an input here: callers pass the arrays.
"""
import numpy as np
import scipy.sparse as sps
from scipy.sparse.linalg import splu

E_CHARGE = 1.602176634e-19
EPS0 = 8.8541878128e-12
M_E = 9.1093837015e-31
AMU = 1.66053906660e-27


def permittivity(solid, mask, p):
    """trench_charging_2d.py:244-248"""
    eps = np.where(solid, p.eps_r, 1.0)
    return np.where(mask, p.mask_eps_r, eps) if p.mask_type == "dielectric" else eps


def poisson_matrix(eps, cond, p):
    """div(eps grad phi) as a sparse matrix (trench_charging_2d.py:252-294)."""
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
    idx = np.arange(nx * ny).reshape(nx, ny)
    rows = [idx.ravel(), idx.ravel(), idx.ravel(), idx[:, :-1].ravel(), idx[:, 1:].ravel()]
    cols = [idx.ravel(), np.roll(idx, -1, axis=0).ravel(), np.roll(idx, 1, axis=0).ravel(),
            idx[:, 1:].ravel(), idx[:, :-1].ravel()]
    vals = [diag.ravel(), ce.ravel(), cw.ravel(), cn[:, :-1].ravel(), cs[:, 1:].ravel()]
    return sps.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(nx * ny, nx * ny)).tocsc()


def make_solver(A, cond):
    """trench_charging_2d.py:297-309"""
    if not cond.any():
        return splu(A).solve
    flat = cond.ravel()
    n_free = int((~flat).sum())
    col = np.where(flat, n_free, np.cumsum(~flat) - 1)
    E = sps.csr_matrix((np.ones(flat.size), (np.arange(flat.size), col)), shape=(flat.size, n_free + 1))
    lu = splu((E.T @ A @ E).tocsc())
    return lambda b: E @ lu.solve(E.T @ b)


def boundary_rhs(p, eps, volts, fixed_sides=True):
    """trench_charging_2d.py:323-337"""
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


def setup_fields(p, solid, mask, circuit=None):
    """trench_charging_2d.py:340-413 (fixed voltages or a circuit waveform dict)."""
    driven = p.field_mode != "floating"
    if p.field_mode in ("circuit", "circuit_rf"):
        t = np.asarray(circuit["t"])
        period = (t[1] - t[0]) * t.size
        if p.field_mode == "circuit":
            at = (p.rf_phase % 360.0) / 360.0 * period
            v = {k: float(np.interp(at, np.append(t, period), np.append(circuit[k], circuit[k][0])))
                 for k in ("uw", "um", "up")}
            volts = dict(substrate=v["uw"] - v["up"], mask=v["um"] - v["up"], top=0.0)
        else:
            wave = np.column_stack((circuit["uw"] - circuit["up"], circuit["um"] - circuit["up"]))
            mean = wave.mean(axis=0)
            volts = dict(substrate=float(mean[0]), mask=float(mean[1]), top=0.0)
    else:
        volts = dict(substrate=p.substrate_voltage, mask=p.mask_voltage, top=p.top_voltage)
    cond = mask if p.mask_type == "conductor" else np.zeros_like(mask)
    eps = permittivity(solid, mask, p)
    A = poisson_matrix(eps, cond, p)
    if driven and cond.any():
        free = ~cond.ravel()
        lu = splu(A[free][:, free].tocsc())

        def solve(b):
            out = np.zeros_like(b, dtype=float)
            out[free] = lu.solve(b[free])
            return out
        phi_cond = cond.ravel().astype(float) * volts["mask"]
        mask_rhs = -(A @ phi_cond)
    else:
        solve = make_solver(A, cond)
        phi_cond = np.zeros(cond.size)
        mask_rhs = np.zeros(cond.size)
    rhs = boundary_rhs(p, eps, volts)
    external = (solve(rhs.ravel() + mask_rhs) + phi_cond).reshape(eps.shape)
    fields = dict(A=A, solve=solve, cond=cond, eps=eps, external=external, boundary_rhs=rhs,
                  volts=volts, floating=bool(cond.any() and not driven), rf=None)
    if p.field_mode == "circuit_rf":
        basis = []
        for vs, vm in ((1.0, 0.0), (0.0, 1.0)):
            brhs = boundary_rhs(p, eps, dict(substrate=vs, mask=vm, top=0.0), fixed_sides=False)
            bc = cond.ravel().astype(float) * vm
            basis.append((solve(brhs.ravel() - A @ bc) + bc).reshape(eps.shape))
        basis = np.array(basis)
        electric = [compute_field(v, ~solid, p, 0.0) for v in basis]
        dt_max = period / p.rf_time_steps
        if p.rf_wave == "pulse":
            dt_max = min(dt_max, p.rf_rise / 8)
        fields["rf"] = dict(period=period, wave=wave - mean, phi=basis,
                            Ex=np.array([v[0] for v in electric]), Ey=np.array([v[1] for v in electric]),
                            dt_max=dt_max)
    return fields


def _grad(c, m, pl, vm, vp, dx):
    """trench_charging_2d.py:429-436"""
    g = np.zeros_like(c)
    both = vm & vp
    g = np.where(both, (pl - m) / (2 * dx), g)
    g = np.where(vp & ~vm, (pl - c) / dx, g)
    g = np.where(vm & ~vp, (c - m) / dx, g)
    return -g


def compute_field(phi, vac, p, top_voltage=None):
    """trench_charging_2d.py:439-454"""
    dx = p.dx
    Ex = _grad(phi, np.roll(phi, 1, 0), np.roll(phi, -1, 0), np.roll(vac, 1, 0), np.roll(vac, -1, 0), dx)
    vtop = p.top_voltage if top_voltage is None else top_voltage
    ghost_top = 2 * vtop - phi[:, -1] if p.top_bc == "dirichlet" else phi[:, -1]
    ghost_bot = 2 * p.substrate_voltage - phi[:, 0]
    pD = np.concatenate([ghost_bot[:, None], phi[:, :-1]], axis=1)
    pU = np.concatenate([phi[:, 1:], ghost_top[:, None]], axis=1)
    f = np.zeros((phi.shape[0], 1), dtype=bool)
    vD = np.concatenate([f, vac[:, :-1]], axis=1)
    vU = np.concatenate([vac[:, 1:], ~f], axis=1)
    Ey = _grad(phi, pD, pU, vD, vU, dx)
    return Ex, Ey


def surface_cells(solid, vacuum=None):
    """trench_charging_2d.py:734-744"""
    nx, ny = solid.shape
    vp = np.pad(~solid if vacuum is None else vacuum, ((0, 0), (1, 1)), constant_values=False)
    near = np.zeros_like(solid)
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            if sx == 0 and sy == 0:
                continue
            near |= np.roll(vp, -sx, axis=0)[:, 1 + sy: 1 + sy + ny]
    return solid & near


def inner_surface_cells(solid, p):
    """trench_charging_2d.py:747-752"""
    inner_vac = ~solid.copy()
    inner_vac[:, :p.floor_t] = False
    inner_vac[:, p.floor_t + p.trench_d + p.mask_t:] = False
    return surface_cells(solid, inner_vac)


def build_leakage(solid, solve, p):
    """trench_charging_2d.py:768-803"""
    nx, ny = solid.shape
    dx = p.dx
    ix, iy = np.nonzero(surface_cells(solid))
    m = ix.size
    smap = -np.ones((nx, ny), dtype=np.int64)
    smap[ix, iy] = np.arange(m)
    g = p.sigma_s / dx
    G = np.zeros((m, m))
    for a, b in ((smap, np.roll(smap, -1, axis=0)), (smap[:, :-1], smap[:, 1:])):
        sel = (a >= 0) & (b >= 0)
        a, b = a[sel], b[sel]
        np.add.at(G, (a, b), g)
        np.add.at(G, (b, a), g)
        np.add.at(G, (a, a), -g)
        np.add.at(G, (b, b), -g)
    flat = ix * ny + iy
    B = np.zeros((nx * ny, m))
    B[flat, np.arange(m)] = -1.0 / (dx ** 2 * EPS0)
    P = solve(B)[flat, :]
    M = np.linalg.inv(np.eye(m) - p.dt_batch * (G @ P))
    cut = p.floor_t + p.trench_d // 2
    region = inner_surface_cells(solid, p)[ix, iy] & (iy < cut)
    return dict(flat=flat, M=M, G=G, region=region)


def conductor_response(solve, cond, dx):
    """trench_charging_2d.py:807-812"""
    b = np.zeros(cond.size)
    b[np.flatnonzero(cond)[0]] = -1.0 / (dx ** 2 * EPS0)
    return solve(b).reshape(cond.shape)


def conductor_step(n_i, n_e, q, C, Te, drift=0.0):
    """trench_charging_2d.py:815-830"""
    x_i, x_e = q * n_i / C + drift, q * n_e / C
    if n_e == 0:
        return x_i
    k = x_i / Te
    frac = -np.expm1(-k) / k if k != 0 else 1.0
    return -Te * np.logaddexp(-k, np.log(x_e / Te * frac))


def opening_span(solid, row):
    """trench_charging_2d.py:229-232"""
    cells = np.flatnonzero(~solid[:, row])
    return int(cells[0]), int(cells[-1] + 1)


class BatchState:
    """State of the reference batch loop between tracer calls.

    Restates the per-batch update of trench_charging_2d.py:1176-1285 for the
    settings the CUDA path covers (floating / fixed field modes; leakage on or
    off).  ``step(cnt_i, cnt_e, esc, lost)`` applies one batch's counts.
    """

    def __init__(self, p, solid, mask, circuit=None):
        self.p = p
        self.solid, self.mask = solid, mask
        self.vac = ~solid
        nx, ny = solid.shape
        self.fields = f = setup_fields(p, solid, mask, circuit)
        self.cond = f["cond"]
        self.solve = f["solve"]
        self.conductor = f["floating"]
        self.driven = p.field_mode != "floating"
        self.wface = np.where(self.cond, 1.0, f["eps"] / (1.0 + f["eps"]))
        self.leak = build_leakage(solid, self.solve, p) if p.sigma_s > 0 else None
        if self.conductor:
            self.g_cond = conductor_response(self.solve, self.cond, p.dx)
            self.C_cond = 1.0 / self.g_cond[self.cond][0]
            self.c_cell = np.flatnonzero(surface_cells(solid) & self.cond)[0]
        w_real = p.flux * (nx * p.dx) * p.dt_batch / p.n_per_batch
        self.q_macro = E_CHARGE * w_real
        self.b0, self.b1 = opening_span(solid, p.floor_t)
        self.e0, self.e1 = opening_span(solid, p.floor_t + p.trench_d + p.mask_t - 1)
        self.rho = np.zeros((nx, ny))
        self.phi = f["external"].copy()
        self.Ex, self.Ey = compute_field(self.phi, self.vac, p, f["volts"]["top"])
        self.hist = dict(ratio_i_bottom=[], ratio_e_bottom=[], esc_e=[], lost=[], leak=[])

    def barrier(self):
        return (self.phi, self.wface) if self.p.wall_model == "barrier" else None

    def step(self, cnt_i, cnt_e, esc, n_lost):
        p, dx = self.p, self.p.dx
        nx, ny = self.rho.shape
        rho = self.rho
        rho_prev = rho.copy() if self.conductor else None
        drho = (cnt_i - cnt_e) * self.q_macro / dx ** 2
        if self.cond.any():
            drho[self.cond] = 0.0
        rho += drho
        leak_ratio = 0.0
        if self.leak is not None:
            leak = self.leak
            Qs = rho.flat[leak["flat"]] * dx ** 2
            Qs_old = Qs
            if np.any(self.fields["external"]):
                Qs = Qs + p.dt_batch * (leak["G"] @ self.fields["external"].ravel()[leak["flat"]])
            Qs_new = leak["M"] @ Qs
            rho.flat[leak["flat"]] = Qs_new / dx ** 2
            dQ = Qs_old[leak["region"]].sum() - Qs_new[leak["region"]].sum()
            leak_ratio = dQ / p.dt_batch / (E_CHARGE * p.flux * (self.e1 - self.e0) * dx)
        if self.driven:
            rho[self.cond] = 0.0
        if self.conductor:
            drift = ((rho - rho_prev) * self.g_cond).sum() * dx ** 2
            dV = conductor_step(cnt_i[self.cond].sum(), cnt_e[self.cond].sum(), self.q_macro,
                                self.C_cond, p.electron_temp_eV, drift)
            rho.flat[self.c_cell] += self.C_cond * (dV - drift) / dx ** 2
        self.phi = self.solve((-rho / EPS0).ravel()).reshape(nx, ny) + self.fields["external"]
        self.Ex, self.Ey = compute_field(self.phi, self.vac, p, self.fields["volts"]["top"])
        frac_open = (self.b1 - self.b0) / nx
        norm = p.n_per_batch * frac_open
        self.hist["ratio_i_bottom"].append(cnt_i[self.b0:self.b1, p.floor_t - 1].sum() / norm)
        self.hist["ratio_e_bottom"].append(cnt_e[self.b0:self.b1, p.floor_t - 1].sum() / norm)
        self.hist["esc_e"].append(esc[1] / p.n_per_batch)
        self.hist["lost"].append(n_lost / (2 * p.n_per_batch))
        self.hist["leak"].append(leak_ratio)
