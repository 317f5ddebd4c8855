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
