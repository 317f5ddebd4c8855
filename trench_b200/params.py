"""Run parameters of the charging step.

``Params`` keeps the reference's field names, meanings and defaults
(trench_charging_2d.py:103-174) so a reference ``Params`` instance and this one
are interchangeable: every function of this package reads parameters by
attribute name only.
"""
from dataclasses import dataclass

E_CHARGE = 1.602176634e-19   # C
EPS0 = 8.8541878128e-12      # F/m
M_E = 9.1093837015e-31       # kg
AMU = 1.66053906660e-27      # kg

MASK_TYPES = ("conductor", "dielectric")
WALL_MODELS = ("barrier", "absorb")
FIELD_MODES = ("floating", "fixed", "circuit", "circuit_rf")
SIDE_BCS = ("periodic", "pillar", "fixed")


@dataclass
class Params:
    # grid and geometry (cells)
    dx: float = 5e-9
    nx: int = 60
    trench_w: int = 20
    trench_offset: int = 0
    trench_taper_deg: float = 0.0
    trench_d: int = 80
    floor_t: int = 10
    n_vac: int = 50
    eps_r: float = 3.9
    top_bc: str = "dirichlet"
    # mask
    mask_t: int = 60
    mask_taper_deg: float = 0.0
    mask_type: str = "conductor"
    mask_eps_r: float = 3.0
    # external potential
    field_mode: str = "floating"
    rf_phase: float = 0.0
    rf_time_steps: int = 256
    substrate_voltage: float = 0.0
    mask_voltage: float = 0.0
    top_voltage: float = 0.0
    side_bc: str = "periodic"
    left_voltage: float = 0.0
    right_voltage: float = 0.0
    # vertical-ion probe
    probe_ions: int = 1000
    probe_energy_eV: float = 100.0
    probe_trajectories: int = 40
    # plasma
    flux: float = 1e20
    ion_mass_amu: float = 40.0
    ion_energy_eV: float = 100.0
    ion_temp_eV: float = 0.5
    electron_temp_eV: float = 3.0
    # RF bias (inputs; the circuit itself is the reference's CPU code)
    bias: str = "rf"
    rf_freq: float = 13.56e6
    rf_volt: float = 100.0
    rf_wave: str = "sine"
    rf_duty: float = 0.1
    rf_rise: float = 1e-9
    c_block: float = 4900e-12
    wafer_d: float = 0.3
    wall_ratio: float = 5.0
    ied_model: str = "sheath"
    gas_pressure: float = 1.0
    gas_temp: float = 300.0
    # surface leakage
    sigma_s: float = 1e-15
    # run to steady charge
    until_steady: bool = False
    max_batches: int = 3000
    steady_window: int = 30
    steady_rtol: float = 0.005
    steady_charge_rtol: float = 0.005
    steady_charge_atol: float = 1e-15
    steady_hold: int = 2
    # numerics
    backend: str = "cpu"
    cuda_device: int = 0
    n_batches: int = 300
    n_per_batch: int = 3000
    dt_batch: float = 1e-4
    cfl: float = 0.35
    max_steps: int = 3000
    wall_model: str = "barrier"
    seed: int = 1


def is_tapered(p):
    """Corner crossing and first-face deposit are on (trench_charging_2d.py:554)."""
    return bool(p.trench_taper_deg or (p.mask_t > 0 and p.mask_taper_deg))
