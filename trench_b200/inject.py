"""Particle injection at the top boundary.

``inject`` draws from the generator in the same order as the reference
(trench_charging_2d.py:458-489), so the same seed gives the same particles.
The samplers below build the ion energy/angle distributions of the benchmark
workloads as ``ion_velocity(rng, n) -> (vx, vy)`` hooks, the form in which the
reference passes its sheath IED/IAD sets (plasma_circuit.py:306-314).
"""
import numpy as np

from .params import AMU, E_CHARGE, M_E


def inject(p, n, ny, rng, ion_energy=None, ion_velocity=None):
    """n ions then n electrons at y = Ly - 1e-3 dx; returns x, y, vx, vy, qm, spc."""
    dx = p.dx
    Lx, Ly = p.nx * dx, ny * dx
    m_i = p.ion_mass_amu * AMU
    xi = rng.uniform(0, Lx, n)
    if ion_velocity is not None:
        vxi, vyi = ion_velocity(rng, n)
    else:
        Ei = p.ion_energy_eV * np.ones(n) if ion_energy is None else ion_energy(rng, n)
        vyi = -np.sqrt(2 * Ei * E_CHARGE / m_i)
        vxi = rng.normal(0, np.sqrt(p.ion_temp_eV * E_CHARGE / m_i), n)
    s = np.sqrt(p.electron_temp_eV * E_CHARGE / M_E)
    xe = rng.uniform(0, Lx, n)
    vxe = rng.normal(0, s, n)
    vye = -s * np.sqrt(-2.0 * np.log(1.0 - rng.uniform(size=n)))
    x = np.concatenate([xi, xe])
    y = np.full(2 * n, Ly - 1e-3 * dx)
    vx = np.concatenate([vxi, vxe])
    vy = np.concatenate([vyi, vye])
    qm = np.concatenate([np.full(n, E_CHARGE / m_i), np.full(n, -E_CHARGE / M_E)])
    spc = np.concatenate([np.zeros(n, dtype=np.int8), np.ones(n, dtype=np.int8)])
    return x, y, vx, vy, qm, spc


def energy_angle_sampler(p, energy, angle):
    """Ion velocities from an energy sampler (eV) and a polar-angle sampler (rad),
    measured from the downward normal: vx = v sin(theta), vy = -v cos(theta)."""
    m_i = p.ion_mass_amu * AMU

    def sample(rng, n):
        e = np.maximum(energy(rng, n), 0.0)
        th = angle(rng, n)
        v = np.sqrt(2 * e * E_CHARGE / m_i)
        return v * np.sin(th), -v * np.cos(th)
    return sample


def gaussian_angle(sigma_deg):
    """Polar angle ~ N(0, sigma)."""
    s = np.radians(sigma_deg)
    return lambda rng, n: rng.normal(0.0, s, n)


def half_gaussian_angle(sigma_deg):
    """|N(0, sigma)| with a random sign (half-Gaussian IAD, both directions)."""
    s = np.radians(sigma_deg)

    def sample(rng, n):
        a = np.abs(rng.normal(0.0, s, n))
        return np.where(rng.random(n) < 0.5, -a, a)
    return sample


def mixture_energy(components):
    """Energy mixture; components = [(weight, kind, a, b)] with kind in
    {"normal" (mean, sigma), "uniform" (lo, hi), "exp" (scale, -)}.  Weights are
    normalised to sum to one."""
    w = np.array([c[0] for c in components], dtype=float)
    w = w / w.sum()

    def sample(rng, n):
        which = rng.choice(len(components), size=n, p=w)
        out = np.empty(n)
        for k, (_, kind, a, b) in enumerate(components):
            sel = which == k
            m = int(sel.sum())
            if kind == "normal":
                out[sel] = rng.normal(a, b, m)
            elif kind == "uniform":
                out[sel] = rng.uniform(a, b, m)
            elif kind == "exp":
                out[sel] = rng.exponential(a, m)
            else:
                raise ValueError(f"unknown energy component {kind!r}")
        return out
    return sample


def launch_times(rng, n, period):
    """Stratified RF launch times over one period, shuffled (trench_rf.py:14-18)."""
    times = (np.arange(n) + rng.random(n)) * period / n
    rng.shuffle(times)
    return times


# ---- device-side injection ---------------------------------------------------------

def philox4x32_10(counters, key):
    """Philox4x32-10 (Salmon et al., SC'11) on the host: counters (n, 4) uint32, key
    (k0, k1) -> (n, 4) uint32.  The device generator of tb_inject computes the same."""
    c = np.array(counters, dtype=np.uint64) & 0xFFFFFFFF
    k0, k1 = np.uint64(key[0] & 0xFFFFFFFF), np.uint64(key[1] & 0xFFFFFFFF)
    m0, m1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
    w0, w1 = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
    mask = np.uint64(0xFFFFFFFF)
    for r in range(10):
        if r:
            k0 = (k0 + w0) & mask
            k1 = (k1 + w1) & mask
        p0 = m0 * c[:, 0]
        p1 = m1 * c[:, 2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & mask
        hi1, lo1 = p1 >> np.uint64(32), p1 & mask
        c = np.stack([hi1 ^ c[:, 1] ^ k0, lo1, hi0 ^ c[:, 3] ^ k1, lo0], axis=1)
    return c.astype(np.uint32)


def histogram_table(edges, weights):
    """Inverse-CDF table (edges, cdf) of a histogram with non-negative bin weights."""
    edges = np.asarray(edges, dtype=np.float64)
    w = np.asarray(weights, dtype=np.float64)
    if edges.ndim != 1 or len(edges) != len(w) + 1 or np.any(np.diff(edges) <= 0):
        raise ValueError("a table needs increasing bin edges, one more than the weights")
    if np.any(w < 0) or not np.isfinite(w).all() or w.sum() <= 0:
        raise ValueError("bin weights must be finite, non-negative and not all zero")
    cdf = np.concatenate([[0.0], np.cumsum(w) / w.sum()])
    cdf[-1] = 1.0
    return edges, cdf


def table_from_pdf(pdf, lo, hi, bins=1024):
    """Histogram table of a density on [lo, hi] (bin-centre values times width)."""
    edges = np.linspace(lo, hi, bins + 1)
    centres = 0.5 * (edges[:-1] + edges[1:])
    return histogram_table(edges, np.maximum(pdf(centres), 0.0) * np.diff(edges))


def bimodal_gaussian_pdf(m1, s1, m2, s2, w1=0.5):
    g = lambda e, m, s: np.exp(-0.5 * ((e - m) / s) ** 2) / (s * np.sqrt(2 * np.pi))
    return lambda e: w1 * g(e, m1, s1) + (1 - w1) * g(e, m2, s2)


def half_gaussian_pdf(sigma):
    return lambda t: np.exp(-0.5 * (t / sigma) ** 2)


class DeviceInjector:
    """Fills a ChargingCase's particle buffers on the GPU each batch (tb_inject).

    energy_table / angle_table: (edges, cdf) from histogram_table or table_from_pdf
    (energy in eV, angle in radians); None uses p.ion_energy_eV / the lateral
    thermal velocity of p.ion_temp_eV like the reference."""

    def __init__(self, case, seed=0, energy_table=None, angle_table=None, angle_random_sign=True, bins=False):
        import ctypes
        import torch
        from . import _capi
        from .params import AMU, E_CHARGE, M_E
        from .tracer import _ptr
        p = case.p
        self.case = case
        dev = case.dev
        f = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
        a = _capi.InjectArgs()
        a.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        a.n_species = int(p.n_per_batch)
        a.d_x, a.d_y, a.d_vx, a.d_vy, a.d_qm = (_ptr(t) for t in case.X)
        a.d_spc = _ptr(case.SPC)
        a.lx = p.nx * p.dx
        a.y0 = case.ny * p.dx - 1e-3 * p.dx
        m_i = p.ion_mass_amu * AMU
        a.qm_ion, a.qm_electron = E_CHARGE / m_i, -E_CHARGE / M_E
        a.ion_mass, a.e_charge = m_i, E_CHARGE
        a.electron_sigma = float(np.sqrt(p.electron_temp_eV * E_CHARGE / M_E))
        a.ion_energy_eV = float(p.ion_energy_eV)
        if p.field_mode in ("circuit", "circuit_rf") and energy_table is None:
            # ions start at the plasma potential with the Bohm energy (trench_charging_2d.py:1135-1139)
            a.ion_energy_eV = float(p.electron_temp_eV) / 2
        a.ion_lateral_sigma = float(np.sqrt(p.ion_temp_eV * E_CHARGE / m_i))
        self._keep = []
        if energy_table is not None:
            e, c = (f(v) for v in energy_table)
            self._keep += [e, c]
            a.d_energy_edges, a.d_energy_cdf, a.n_energy = _ptr(e), _ptr(c), len(energy_table[0]) - 1
        if angle_table is not None:
            e, c = (f(v) for v in angle_table)
            self._keep += [e, c]
            a.d_angle_edges, a.d_angle_cdf, a.n_angle = _ptr(e), _ptr(c), len(angle_table[0]) - 1
        a.angle_random_sign = int(bool(angle_random_sign))
        if case.rf is not None:
            # circuit_rf: stratified launch times over one period into the case's clock
            a.d_clock, a.period = _ptr(case.clock), float(case.rf["period"])
        self.bin_e = self.bin_a = None
        if bins:
            # table bin of every ion's energy and angle (the adjoint's histories)
            self.bin_e = torch.zeros(int(p.n_per_batch), dtype=torch.uint16, device=dev)
            self.bin_a = torch.zeros(int(p.n_per_batch), dtype=torch.uint16, device=dev)
            a.d_bin_e, a.d_bin_a = _ptr(self.bin_e), _ptr(self.bin_a)
        self.args = a
        self._ctypes = ctypes
        self._capi = _capi

    def __call__(self, batch=None):
        """Inject on the current stream: batch number `batch` (the Philox counter), or
        with batch=None the case's own device batch counter + 1, so a captured CUDA
        graph draws a fresh batch on every replay."""
        import torch
        from .tracer import _ptr
        case = self.case
        if 2 * self.args.n_species > case.capacity:
            raise ValueError("the case buffers hold fewer particles than one batch")
        if batch is None:
            self.args.batch = 0
            self.args.d_counter = _ptr(case.batch)
        else:
            self.args.batch = int(batch)
            self.args.d_counter = None
        s = self._ctypes.c_void_p(torch.cuda.current_stream(case.dev).cuda_stream)
        case.ctx.check(self._capi.lib().tb_inject(case.ctx.handle, self._ctypes.byref(self.args), s))
        case.n_loaded = 2 * int(self.args.n_species)
