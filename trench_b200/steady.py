"""Steady-state stopping of the charging loop (``until_steady``).

The stopping rule is the reference's (trench_charging_2d.py:846-947, 1302-1320):
every ``steady_window`` (W) batches, once two windows of history exist, the last
window of every potential probe is compared with the window before it, and so is
every charge monitor together with its net drift over a window; after
``steady_hold`` consecutive passes the run has converged.  A window's mean is
compared through a standard error that (1) removes the window's linear trend and
(2) shrinks the sample size by the lag-1 autocorrelation of what is left (an AR(1)
effective size n (1 - r1) / (1 + r1), r1 clipped to [0, 0.95]).

Here every check runs over all probes (or monitors) at once: the histories are
stacked into one (series, samples) array and the window statistics are closed-form
row reductions -- the trend is the least-squares line about the window's centre
time, the autocorrelation the Pearson coefficient of the residual against itself one
batch later.

The monitors are summed on the GPU every batch (tb_step_monitors); the checks run
on the host every W batches over the history read back once.
"""
import numpy as np

from . import geometry


def charge_monitors(solid, mask, i0, i1, p):
    """Flat cell indices of each charge monitor (trench_charging_2d.py:850-868): the
    left and right inner sidewalls of the dielectric (split at the interface opening's
    centre), the cells under the trench floor's opening, the exposed dielectric
    surface, each sidewall in three height bands, and the mask."""
    nx, ny = solid.shape
    col, row = np.indices(solid.shape)
    in_trench_rows = (row >= p.floor_t) & (row < p.floor_t + p.trench_d)
    inner_wall = geometry.inner_surface_cells(solid, p) & in_trench_rows
    left_half = col + 0.5 < (i0 + i1) / 2
    lo, hi = geometry.opening_span(solid, p.floor_t)
    floor = np.zeros_like(solid)
    floor[lo:hi, p.floor_t - 1] = True
    exposed = geometry.surface_cells(solid)
    if p.mask_type == "conductor":
        exposed = exposed & ~mask
    sides = {"left": inner_wall & left_half, "right": inner_wall & ~left_half}
    regions = {**sides, "bottom": floor, "surface": exposed}
    # three bands of trench rows, the first (lowest) bands one row longer when the depth
    # does not divide by three
    bands = np.array_split(np.arange(p.floor_t, p.floor_t + p.trench_d), 3)
    for side, cells in sides.items():
        for k, band in enumerate(bands, start=1):
            if band.size:
                regions[f"{side} band {k}"] = cells & (row >= band[0]) & (row <= band[-1])
    if mask.any():
        regions["mask"] = mask
    return {name: np.flatnonzero(r) for name, r in regions.items()}


def _window_stats(X):
    """Mean and trend/autocorrelation-corrected standard error of each row of X
    (series, samples)."""
    X = np.atleast_2d(np.asarray(X, dtype=float))
    n = X.shape[1]
    tc = np.arange(n) - 0.5 * (n - 1)          # sample times about the window centre
    mean = X.mean(axis=1)
    slope = (X - mean[:, None]) @ tc / (tc @ tc)
    resid = X - mean[:, None] - slope[:, None] * tc
    resid_c = resid - resid.mean(axis=1, keepdims=True)
    var = (resid_c ** 2).sum(axis=1) / (n - 2)
    a, b = resid[:, :-1], resid[:, 1:]
    a = a - a.mean(axis=1, keepdims=True)
    b = b - b.mean(axis=1, keepdims=True)
    with np.errstate(invalid="ignore", divide="ignore"):
        r1 = (a * b).sum(axis=1) / np.sqrt((a * a).sum(axis=1) * (b * b).sum(axis=1))
    r1 = np.where((var > 0) & np.isfinite(r1), np.clip(r1, 0.0, 0.95), 0.0)
    n_eff = np.maximum(n * (1 - r1) / (1 + r1), 1.0)
    return mean, np.sqrt(var / n_eff)


def mean_and_se(x):
    """(mean, standard error) of one window (trench_charging_2d.py:877-890)."""
    m, se = _window_stats(x)
    return float(m[0]), float(se[0])


def check_steady(hist, probes, p, reference=None):
    """Probe potentials (trench_charging_2d.py:893-914): |last window mean - previous
    window mean| <= max(steady_rtol x the largest last-window potential (measured from
    `reference` when given, at least 1 V), 3 standard errors of the difference) for every
    probe.  Returns (ok, the probe furthest from passing, its difference, its tolerance)."""
    W = p.steady_window
    names = list(probes)
    H = np.array([np.asarray(hist[k], dtype=float)[-2 * W:] for k in names])
    m_new, se_new = _window_stats(H[:, W:])
    m_old, se_old = _window_stats(H[:, :W])
    base = np.array([reference[k] for k in names]) if reference is not None else 0.0
    scale = max(1.0, float(np.max(np.abs(m_new - base))))
    d = m_new - m_old
    tol = np.maximum(p.steady_rtol * scale, 3.0 * np.hypot(se_new, se_old))
    worst = int(np.argmax(np.abs(d) / tol))
    return bool(np.all(np.abs(d) <= tol)), names[worst], float(d[worst]), float(tol[worst])


def check_charge_steady(charge_hist, p):
    """Charge monitors (trench_charging_2d.py:917-945), two tests per monitor over the
    last two windows: the window means (tolerance max(atol, rtol x the larger |mean|,
    3 standard errors)) and the net drift of one window from the batch-to-batch
    changes (tolerance max(atol, 3 standard errors); a steadily charging surface fails
    it however large its charge).  Returns the test furthest from passing as a dict
    (name, kind, d, tol, ratio, rate in C/m/s, unit) with ``ok`` for all of them."""
    W = p.steady_window
    rtol, atol, dt = p.steady_charge_rtol, p.steady_charge_atol, p.dt_batch
    if not (np.isfinite(rtol) and rtol > 0 and np.isfinite(atol) and atol >= 0 and W >= 5
            and np.isfinite(dt) and dt > 0):
        raise ValueError("the charge check needs rtol > 0, atol >= 0 (finite), dt_batch > 0 and a window of "
                         "at least 5 batches")
    names = list(charge_hist)
    if not names or min(len(v) for v in charge_hist.values()) < 2 * W:
        raise ValueError("the charge check needs two windows of history for every monitor")
    Q = np.array([np.asarray(charge_hist[k], dtype=float)[-2 * W:] for k in names])
    if Q.ndim != 2 or not np.isfinite(Q).all():
        raise ValueError("the charge history holds non-finite values")
    m_new, se_new = _window_stats(Q[:, W:])
    m_old, se_old = _window_stats(Q[:, :W])
    rate, se_rate = _window_stats(np.diff(Q, axis=1))
    d = np.stack([m_new - m_old, rate * W], axis=1)
    tol = np.stack([np.maximum.reduce([np.full(len(names), atol), rtol * np.maximum(np.abs(m_new), np.abs(m_old)),
                                       3 * np.hypot(se_new, se_old)]),
                    np.maximum(atol, 3 * se_rate * W)], axis=1)
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.where(tol > 0, np.abs(d) / tol, np.where(d == 0, 0.0, np.inf))
    k, kind = divmod(int(np.argmax(ratio)), 2)
    return dict(name=names[k], kind=("mean", "drift")[kind], d=float(d[k, kind]), tol=float(tol[k, kind]),
                ratio=float(ratio[k, kind]), rate=float(rate[k] / dt), unit="C/m",
                ok=bool(np.all(np.abs(d) <= tol)))


def history_start(hist, probes, charge_hist):
    """First batch from which every probe and monitor history is finite (a resumed run
    whose saved results lack some of them carries NaN there)."""
    series = [np.asarray(hist[k], dtype=float) for k in probes] + \
             [np.asarray(v, dtype=float) for v in charge_hist.values()]
    last_bad = [np.flatnonzero(~np.isfinite(s))[-1] + 1 for s in series if not np.isfinite(s).all()]
    return int(max(last_bad, default=0))
