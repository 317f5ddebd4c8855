"""Staircase trench geometry and the cell sets the charging step uses.

Host-side setup, run once per case.  The trench is described by its continuous
outline -- a centre line and, per layer (dielectric below the mask interface,
mask above it), a half-width that grows linearly with height by the layer's taper
-- and rasterised row by row: a cell is vacuum when its centre lies in the half-
open interval [centre - half-width, centre + half-width) of its row.  Each row's
opening is therefore one contiguous span of columns, found by a binary search of
the column centres against the two ends of the interval; the solid/mask arrays,
the wall columns and the probe cells are all read off these spans.

The rasterisation rule, the validity conditions and the named probe cells are
those of the reference (trench_charging_2d.py:178-248, 734-752, 1153-1166), so
the arrays are the same cell for cell; the construction is this module's own.
"""
from dataclasses import dataclass

import numpy as np

from .params import MASK_TYPES

_CELL_COUNTS = ("nx", "trench_w", "trench_offset", "trench_d", "floor_t", "n_vac", "mask_t")


def opening_widths(p):
    """Continuous opening width (cells) at the trench bottom, at the dielectric/mask
    interface (the width's reference level) and at the mask top
    (trench_charging_2d.py:178-182)."""
    grow = lambda depth, deg: 2.0 * depth * np.tan(np.radians(deg))
    return dict(bottom=p.trench_w - grow(p.trench_d, p.trench_taper_deg), interface=float(p.trench_w),
                top=p.trench_w + grow(p.mask_t, p.mask_taper_deg))


def _check(p):
    """Raises ValueError when the parameters do not describe a trench that fits the
    domain with at least one solid column on each side of every opening."""
    counts = [getattr(p, k) for k in _CELL_COUNTS]
    if not all(isinstance(v, (int, np.integer)) for v in counts):
        raise ValueError("geometry sizes are whole numbers of cells")
    if p.nx < 3 or p.trench_w < 1 or p.trench_w > p.nx - 2:
        raise ValueError(f"the trench width must lie in [1, nx - 2] cells (nx={p.nx}, trench_w={p.trench_w})")
    if min(p.floor_t, p.trench_d, p.n_vac) < 1:
        raise ValueError("floor_t, trench_d and n_vac must each be at least one cell")
    left = (p.nx - p.trench_w) // 2 + p.trench_offset
    if left < 1 or left + p.trench_w > p.nx - 1:
        raise ValueError(f"trench_offset={p.trench_offset} leaves no solid column beside the trench")
    if p.mask_t < 0:
        raise ValueError(f"the mask thickness must not be negative (mask_t={p.mask_t})")
    if p.mask_type not in MASK_TYPES:
        raise ValueError(f"unknown mask_type {p.mask_type!r}; expected one of {MASK_TYPES}")
    for key in ("trench_taper_deg", "mask_taper_deg"):
        a = getattr(p, key)
        if not (np.isfinite(a) and abs(a) < 90):
            raise ValueError(f"{key}={a}: a taper is a finite angle strictly between -90 and 90 degrees")
    centre = left + p.trench_w / 2
    for where, w in opening_widths(p).items():
        if w < 1:
            raise ValueError(f"the opening at the {where} is under one cell wide ({w:.3g})")
        if not (1 <= centre - w / 2 and centre + w / 2 <= p.nx - 1):
            raise ValueError(f"the opening at the {where} reaches the domain's side columns")
    return left


@dataclass
class TrenchRaster:
    """The rasterised trench: per grid row the span [lo, hi) of vacuum columns."""
    nx: int
    ny: int
    floor_t: int
    top_ox: int          # first mask row (top of the dielectric)
    top: int             # first row above the mask (vacuum everywhere from here up)
    i0: int              # opening columns at the interface level: [i0, i1)
    i1: int
    lo: np.ndarray       # (ny,) first vacuum column of each row (nx for all-solid rows)
    hi: np.ndarray       # (ny,) one past the last vacuum column (nx for all-solid rows)

    @classmethod
    def of(cls, p):
        i0 = _check(p)
        top_ox = p.floor_t + p.trench_d
        top = top_ox + p.mask_t
        ny = top + p.n_vac
        lo = np.full(ny, p.nx, dtype=np.int64)
        hi = np.full(ny, p.nx, dtype=np.int64)
        lo[top:] = 0
        rows = np.arange(p.floor_t, top)
        yc = rows + 0.5
        # half-width of the opening at each row's centre height, tapered per layer
        slope = np.where(yc < top_ox, np.tan(np.radians(p.trench_taper_deg)), np.tan(np.radians(p.mask_taper_deg)))
        half = p.trench_w / 2 + (yc - top_ox) * slope
        centre = (2 * i0 + p.trench_w) / 2
        xc = np.arange(p.nx) + 0.5
        # the columns whose centre satisfies centre - half <= xc < centre + half
        lo[rows] = np.searchsorted(xc, centre - half, side="left")
        hi[rows] = np.searchsorted(xc, centre + half, side="left")
        return cls(p.nx, ny, p.floor_t, top_ox, top, i0, i0 + p.trench_w, lo, hi)

    def solid(self):
        col = np.arange(self.nx)[:, None]
        return (col < self.lo[None, :]) | (col >= self.hi[None, :])

    def mask(self, solid):
        m = solid.copy()
        m[:, :self.top_ox] = False
        return m


def build_geometry(p):
    """(solid[ix, iy], mask[ix, iy], i0, i1): solid and mask cells (iy = 0 at the
    substrate) and the interface opening [i0, i1); the same arrays as the reference's
    build_geometry (trench_charging_2d.py:185-226).  ValueError for a trench that
    does not fit."""
    r = TrenchRaster.of(p)
    solid = r.solid()
    return solid, r.mask(solid), r.i0, r.i1


def opening_span(solid, row):
    """[left, right) of the vacuum columns of one row (trench_charging_2d.py:229-232)."""
    cols = np.nonzero(~solid[:, row])[0]
    return int(cols.min()), int(cols.max()) + 1


def wall_bounds(solid, p):
    """For every row of the trench and mask (floor_t <= iy < floor_t + trench_d +
    mask_t): the solid column just left of the opening and the one just right of it,
    and the rows (trench_charging_2d.py:235-241)."""
    rows = np.arange(p.floor_t, p.floor_t + p.trench_d + p.mask_t)
    spans = np.array([opening_span(solid, r) for r in rows]).reshape(-1, 2)
    return spans[:, 0] - 1, spans[:, 1], rows


def permittivity(solid, mask, p):
    """Relative permittivity per cell: 1 in vacuum, eps_r in the dielectric, mask_eps_r
    in a dielectric mask (trench_charging_2d.py:244-248)."""
    eps = np.ones(solid.shape)
    eps[solid] = p.eps_r
    if p.mask_type == "dielectric":
        eps[mask] = p.mask_eps_r
    return eps


def surface_cells(solid, vacuum=None):
    """Solid cells with at least one vacuum cell among their 8 neighbours, x periodic
    and rows beyond the grid counted as solid (trench_charging_2d.py:734-744).  The
    3 x 3 neighbourhood test is a separable dilation of the vacuum: along x by the
    periodic shifts, then along y with no wrap."""
    vac = ~solid if vacuum is None else np.asarray(vacuum, dtype=bool)
    along_x = vac | np.roll(vac, 1, axis=0) | np.roll(vac, -1, axis=0)
    near = along_x.copy()
    near[:, 1:] |= along_x[:, :-1]
    near[:, :-1] |= along_x[:, 1:]
    return solid & near


def inner_surface_cells(solid, p):
    """Surface cells exposed to the opening of the trench and mask (the rows between
    the floor and the mask top), the outer top surface excluded
    (trench_charging_2d.py:747-752)."""
    inside = ~solid
    inside[:, :p.floor_t] = False
    inside[:, p.floor_t + p.trench_d + p.mask_t:] = False
    return surface_cells(solid, inside)


def probe_cells(solid, p, conductor_mask):
    """Cells whose potential the history records, by name
    (trench_charging_2d.py:1153-1166): the mask top ten columns left of the
    opening, the mask sidewall at mid-height (dielectric mask only), the left
    sidewall near its top, middle and bottom, the trench floor below the opening
    centre, and the right sidewall at the same three heights."""
    top_ox = p.floor_t + p.trench_d
    top = top_ox + p.mask_t
    left, right, _ = wall_bounds(solid, p)

    def wall(col, row):
        return int(col[row - p.floor_t]), row

    heights = dict(upper=max(p.floor_t, top_ox - 4), middle=p.floor_t + p.trench_d // 2,
                   lower=min(top_ox - 1, p.floor_t + 3))
    mouth, _ = opening_span(solid, top - 1)
    floor_lo, floor_hi = opening_span(solid, p.floor_t)
    probes = {"mask top": (max(0, mouth - 10), top - 1)}
    if p.mask_t > 0 and not conductor_mask:
        probes["mask sidewall"] = wall(left, top_ox + p.mask_t // 2)
    probes.update({f"sidewall {k}": wall(left, y) for k, y in heights.items()})
    probes["bottom center"] = ((floor_lo + floor_hi) // 2, p.floor_t - 1)
    probes.update({f"right sidewall {k}": wall(right, y) for k, y in heights.items()})
    return probes
