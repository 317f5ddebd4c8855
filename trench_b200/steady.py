"""Steady-state stopping of the charging loop (``until_steady``).

Restates the reference's stopping rule (trench_charging_2d.py:1216-1229, 1302-1320):
every ``steady_window`` (W) batches, once 2 W batches of history exist, the mean of
each potential probe over the last W batches is compared with the W before it, and
so is every charge monitor together with its net drift; after ``steady_hold``
consecutive passes the run has converged.

  charge_monitors       trench_charging_2d.py:850-868  (cells summed per monitor)
  mean_and_se           trench_charging_2d.py:877-890  (trend-removed, AR(1)-corrected)
  check_steady          trench_charging_2d.py:893-914
  check_charge_steady   trench_charging_2d.py:917-945
  history_start         trench_charging_2d.py:1034-1041

The monitors themselves are summed on the GPU every batch (tb_step_monitors); the
checks run on the host every W batches over the history read back once.
"""
import numpy as np

from . import geometry


def charge_monitors(solid, mask, i0, i1, p):
    """Cells of each charge monitor: left / right inner sidewall, bottom, the exposed
    dielectric surface, three depth bands per sidewall and the mask (flat indices)."""
    exposed = geometry.surface_cells(solid)
    dielectric = exposed & ~(mask if p.mask_type == "conductor" else np.zeros_like(mask))
    ix, iy = np.indices(solid.shape)
    wall = (iy >= p.floor_t) & (iy < p.floor_t + p.trench_d)
    inner = geometry.inner_surface_cells(solid, p)
    center = (i0 + i1) / 2
    b0, b1 = geometry.opening_span(solid, p.floor_t)
    regions = dict(left=(ix + 0.5 < center) & wall & inner,
                   right=(ix + 0.5 >= center) & wall & inner,
                   bottom=(ix >= b0) & (ix < b1) & (iy == p.floor_t - 1), surface=dielectric)
    for side in ("left", "right"):
        for band, cells in enumerate(np.array_split(np.arange(p.floor_t, p.floor_t + p.trench_d), 3)):
            if len(cells):
                regions[f"{side} band {band + 1}"] = regions[side] & np.isin(iy, cells)
    if mask.any():
        regions["mask"] = mask
    return {key: np.flatnonzero(region) for key, region in regions.items()}


def mean_and_se(x):
    """Mean of a block and its standard error: the variance of the residual after a
    linear fit, with the effective sample size n (1 - r1) / (1 + r1) of the residual's
    lag-1 autocorrelation r1 (clipped to [0, 0.95])."""
    x = np.asarray(x, dtype=float)
    n = x.size
    t = np.arange(n)
    resid = x - np.polyval(np.polyfit(t, x, 1), t)
    var = resid.var(ddof=2)
    r1 = 0.0
    if var > 0:
        r1 = np.corrcoef(resid[:-1], resid[1:])[0, 1]
        r1 = float(np.clip(r1, 0.0, 0.95)) if np.isfinite(r1) else 0.0
    n_eff = max(n * (1 - r1) / (1 + r1), 1.0)
    return x.mean(), np.sqrt(var / n_eff)


def check_steady(hist, probes, p, reference=None):
    """Probe potentials: |mean of the last W - mean of the W before| <= max(rtol x the
    largest probe potential (relative to `reference`), 3 x the combined standard error)
    for every probe.  Returns (ok, worst probe, its difference, its tolerance)."""
    W = p.steady_window
    stats = {k: (mean_and_se(np.asarray(hist[k][-W:])), mean_and_se(np.asarray(hist[k][-2 * W:-W])))
             for k in probes}
    scale = max(1.0, max(abs(c[0] - (reference[k] if reference is not None else 0.0))
                         for k, (c, _) in stats.items()))
    ok, worst = True, (None, 0.0, 1.0, -1.0)
    for k, ((m_c, se_c), (m_p, se_p)) in stats.items():
        d = m_c - m_p
        tol = max(p.steady_rtol * scale, 3.0 * np.hypot(se_c, se_p))
        ok &= abs(d) <= tol
        if abs(d) / tol > worst[3]:
            worst = (k, d, tol, abs(d) / tol)
    return ok, worst[0], worst[1], worst[2]


def check_charge_steady(charge_hist, p):
    """Charge monitors: the difference of the block means (tolerance max(atol, rtol x
    charge, 3 standard errors)) and the net drift over a block from the per-batch
    changes (tolerance max(atol, 3 standard errors)).  Returns the worst check as a
    dict (name, kind, d, tol, ratio, rate, unit) with `ok` for all of them."""
    W = p.steady_window
    if (not np.isfinite(p.steady_charge_rtol) or p.steady_charge_rtol <= 0
            or not np.isfinite(p.steady_charge_atol) or p.steady_charge_atol < 0
            or W < 5 or not np.isfinite(p.dt_batch) or p.dt_batch <= 0):
        raise ValueError("the charge tolerances and batch time must be finite and positive (atol >= 0), "
                         "and the window at least 5")
    if not charge_hist or any(len(q) < 2 * W for q in charge_hist.values()):
        raise ValueError("the charge check needs two windows of history")
    ok, worst = True, None
    for key, values in charge_hist.items():
        q = np.asarray(values[-2 * W:], dtype=float)
        if q.ndim != 1 or not np.isfinite(q).all():
            raise ValueError("the charge history must be finite")
        cur, se_cur = mean_and_se(q[-W:])
        prev, se_prev = mean_and_se(q[:W])
        difference = float(cur - prev)
        mean_tol = max(p.steady_charge_atol, p.steady_charge_rtol * max(abs(cur), abs(prev)),
                       3 * np.hypot(se_cur, se_prev))
        current, se_current = mean_and_se(np.diff(q))
        drift = float(current * W)
        drift_tol = max(p.steady_charge_atol, float(3 * se_current * W))
        for kind, d, tol in (("mean", difference, mean_tol), ("drift", drift, drift_tol)):
            passed = abs(d) <= tol
            ratio = abs(d) / tol if tol > 0 else (0.0 if d == 0 else np.inf)
            ok &= passed
            if worst is None or ratio > worst["ratio"]:
                worst = dict(name=key, kind=kind, d=d, tol=float(tol), ratio=float(ratio),
                             rate=float(current / p.dt_batch), unit="C/m")
    return {**worst, "ok": bool(ok)}


def history_start(hist, probes, charge_hist):
    """First batch after which every probe and monitor history is finite (a resumed
    run whose saved results lack some of them carries NaN there)."""
    first = 0
    for values in [*(hist[k] for k in probes), *charge_hist.values()]:
        missing = np.flatnonzero(~np.isfinite(values))
        if missing.size:
            first = max(first, int(missing[-1]) + 1)
    return first
