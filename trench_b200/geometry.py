"""Staircase trench geometry and the cell sets the charging step uses.

Host-side setup, run once per case.  Each function restates the reference
function cited in its docstring and returns the same arrays.
"""
import numpy as np

from .params import MASK_TYPES


def opening_widths(p):
    """trench_charging_2d.py:178-182"""
    return dict(bottom=p.trench_w - 2 * p.trench_d * np.tan(np.radians(p.trench_taper_deg)),
                interface=float(p.trench_w),
                top=p.trench_w + 2 * p.mask_t * np.tan(np.radians(p.mask_taper_deg)))


def build_geometry(p):
    """solid[ix, iy], mask[ix, iy], i0, i1 (trench_charging_2d.py:185-226).

    A cell is vacuum when its centre lies inside the (tapered) opening.  Raises
    ValueError for the same invalid shapes as the reference.
    """
    ints = ("nx", "trench_w", "trench_offset", "trench_d", "floor_t", "n_vac", "mask_t")
    if (any(not isinstance(getattr(p, k), (int, np.integer)) for k in ints) or p.nx < 3
            or not 1 <= p.trench_w <= p.nx - 2 or min(p.floor_t, p.trench_d, p.n_vac) < 1):
        raise ValueError("geometry cell counts must be positive integers and trench_w <= nx-2")
    i0 = (p.nx - p.trench_w) // 2 + p.trench_offset
    i1 = i0 + p.trench_w
    if i0 < 1 or i1 > p.nx - 1:
        raise ValueError("the shifted trench must leave at least one solid column on each side")
    if p.mask_t < 0:
        raise ValueError(f"mask_t must be >= 0: {p.mask_t}")
    if p.mask_type not in MASK_TYPES:
        raise ValueError(f"mask_type must be one of {MASK_TYPES}: {p.mask_type!r}")
    for key in ("trench_taper_deg", "mask_taper_deg"):
        angle = getattr(p, key)
        if not np.isfinite(angle) or not -90 < angle < 90:
            raise ValueError(f"{key}: taper angle must be finite and within (-90, 90) degrees")
    center = (i0 + i1) / 2
    for level, width in opening_widths(p).items():
        if width < 1:
            raise ValueError(f"opening at the {level} is narrower than one cell")
        if center - width / 2 < 1 or center + width / 2 > p.nx - 1:
            raise ValueError(f"taper at the {level} leaves the domain")
    top_ox = p.floor_t + p.trench_d
    ny = top_ox + p.mask_t + p.n_vac
    solid = np.zeros((p.nx, ny), dtype=bool)
    solid[:, :top_ox + p.mask_t] = True
    y = np.arange(p.floor_t, top_ox + p.mask_t) + 0.5
    slope = np.tan(np.radians(np.where(y < top_ox, p.trench_taper_deg, p.mask_taper_deg)))
    half_width = p.trench_w / 2 + (y - top_ox) * slope
    x = (np.arange(p.nx) + 0.5)[:, None]
    opening = (x >= center - half_width) & (x < center + half_width)
    solid[:, p.floor_t:top_ox + p.mask_t] = ~opening
    mask = solid.copy()
    mask[:, :top_ox] = False
    return solid, mask, i0, i1


def opening_span(solid, row):
    """[left, right) of the vacuum opening in one row (trench_charging_2d.py:229-232)."""
    cells = np.flatnonzero(~solid[:, row])
    return int(cells[0]), int(cells[-1] + 1)


def wall_bounds(solid, p):
    """Solid columns left/right of the opening per row (trench_charging_2d.py:235-241)."""
    iy = np.arange(p.floor_t, p.floor_t + p.trench_d + p.mask_t)
    vac = ~solid[:, iy]
    left = np.argmax(vac, axis=0) - 1
    right = solid.shape[0] - np.argmax(vac[::-1], axis=0)
    return left, right, iy


def permittivity(solid, mask, p):
    """Relative permittivity per cell (trench_charging_2d.py:244-248)."""
    eps = np.where(solid, p.eps_r, 1.0)
    return np.where(mask, p.mask_eps_r, eps) if p.mask_type == "dielectric" else eps


def surface_cells(solid, vacuum=None):
    """Solid cells with a vacuum 8-neighbour; x periodic, rows outside are solid
    (trench_charging_2d.py:734-744)."""
    nx, ny = solid.shape
    vp = np.pad(~solid if vacuum is None else vacuum, ((0, 0), (1, 1)), constant_values=False)
    near = np.zeros_like(solid)
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            if sx or sy:
                near |= np.roll(vp, -sx, axis=0)[:, 1 + sy: 1 + sy + ny]
    return solid & near


def inner_surface_cells(solid, p):
    """trench_charging_2d.py:747-752"""
    inner_vac = ~solid.copy()
    inner_vac[:, :p.floor_t] = False
    inner_vac[:, p.floor_t + p.trench_d + p.mask_t:] = False
    return surface_cells(solid, inner_vac)


def probe_cells(solid, p, conductor_mask):
    """Potential probe cells of the history (trench_charging_2d.py:1153-1166)."""
    top_ox = p.floor_t + p.trench_d
    left, right, _ = wall_bounds(solid, p)
    b0, b1 = opening_span(solid, p.floor_t)
    e0, _ = opening_span(solid, p.floor_t + p.trench_d + p.mask_t - 1)
    probes = {"mask top": (max(0, e0 - 10), top_ox + p.mask_t - 1)}
    if p.mask_t > 0 and not conductor_mask:
        y_mask = top_ox + p.mask_t // 2
        probes["mask sidewall"] = (int(left[y_mask - p.floor_t]), y_mask)
    for level, y_wall in (("upper", max(p.floor_t, top_ox - 4)),
                          ("middle", p.floor_t + p.trench_d // 2),
                          ("lower", min(top_ox - 1, p.floor_t + 3))):
        probes[f"sidewall {level}"] = (int(left[y_wall - p.floor_t]), y_wall)
    probes["bottom center"] = ((b0 + b1) // 2, p.floor_t - 1)
    for level in ("upper", "middle", "lower"):
        y_wall = probes[f"sidewall {level}"][1]
        probes[f"right sidewall {level}"] = (int(right[y_wall - p.floor_t]), y_wall)
    return probes
