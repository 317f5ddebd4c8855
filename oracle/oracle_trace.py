"""ORACLE -- test infrastructure only (the checker, never the product).

Python front end of the scalar FP64 C restatement of the reference CPU tracer
(``trace_oracle.c``).  ``trace`` has the exact call signature and return value of
the reference ``trace_cpu`` (trench_charging_2d.py:542-702) and fills ``record``
the same way (trench_charging_2d.py:565-577, 652-701).  ``trace_detail`` also
returns per-particle status, absorbing cell and step count, which the parity
tests compare with the CUDA path.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_f64 = ctypes.POINTER(ctypes.c_double)
_i32 = ctypes.POINTER(ctypes.c_int32)
_i8 = ctypes.POINTER(ctypes.c_int8)
_u8 = ctypes.POINTER(ctypes.c_uint8)
_lib_handle = None


def build():
    """Compile liboracle.so with the committed Makefile (gcc, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib_handle
    if _lib_handle is None:
        if not LIB.exists():
            build()
        h = ctypes.CDLL(str(LIB))
        h.oracle_trace.restype = ctypes.c_int
        h.oracle_trace.argtypes = [
            ctypes.c_int64, _f64, _f64, _f64, _f64, _f64,
            _f64, _f64, _u8, ctypes.c_int, ctypes.c_int,
            ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
            _f64, _f64,
            _f64, _f64, _f64,
            _f64, ctypes.c_int, ctypes.c_double, ctypes.c_double,
            ctypes.c_double, ctypes.c_double, _f64, _f64,
            ctypes.c_int, _f64, _i32, _f64,
            _i32, ctypes.c_int,
            _i8, _i32, _i32, ctypes.c_int]
        _lib_handle = h
    return _lib_handle


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def default_threads():
    return max(1, len(os.sched_getaffinity(0)))


def is_tapered(p):
    """trench_charging_2d.py:554"""
    return bool(p.trench_taper_deg or (p.mask_t > 0 and p.mask_taper_deg))


def selected_paths(n, count):
    """Indices of the recorded trajectories (trench_charging_2d.py:567)."""
    return np.unique(np.linspace(0, n - 1, min(count, n), dtype=int))


def trace_detail(x, y, vx, vy, qm, Ex, Ey, vac, p, barrier=None, rf=None, record=False,
                 path_count=0, threads=None):
    """Trace copies of the particles; returns a dict of per-particle results."""
    n = len(x)
    nx, ny = vac.shape
    f = lambda a: np.ascontiguousarray(a, dtype=np.float64).copy()
    x, y, vx, vy, qm = f(x), f(y), f(vx), f(vy), f(qm)
    ex = np.ascontiguousarray(Ex, dtype=np.float64)
    ey = np.ascontiguousarray(Ey, dtype=np.float64)
    v8 = np.ascontiguousarray(vac, dtype=np.uint8)
    phi = wface = None
    if barrier is not None:
        phi = np.ascontiguousarray(barrier[0], dtype=np.float64)
        wface = np.ascontiguousarray(barrier[1], dtype=np.float64)
    rf_ex = rf_ey = rf_phi = wave = clock = elapsed = None
    n_phase, period, dt_max, bvs, bvm = 0, 1.0, 1.0, 0.0, 0.0
    if rf is not None:
        rf_ex = np.ascontiguousarray(rf["Ex"], dtype=np.float64)
        rf_ey = np.ascontiguousarray(rf["Ey"], dtype=np.float64)
        rf_phi = np.ascontiguousarray(rf["phi"], dtype=np.float64)
        wave = np.ascontiguousarray(rf["wave"], dtype=np.float64)
        n_phase, period, dt_max = len(wave), float(rf["period"]), float(rf["dt_max"])
        bvs, bvm = (float(v) for v in np.abs(rf["wave"]).max(axis=0))
        clock = np.asarray(rf["initial_time"], dtype=np.float64) % period
        elapsed = np.zeros(n)
    endpoints = np.column_stack((x, y)).astype(np.float64) if record else None
    stride = p.max_steps + 1
    sel = selected_paths(n, path_count) if (record and path_count > 0) else np.zeros(0, int)
    slots = np.full(n, -1, dtype=np.int32)
    slots[sel] = np.arange(sel.size, dtype=np.int32)
    paths = np.zeros((max(sel.size, 1), stride, 2))
    plen = np.ones(max(sel.size, 1), dtype=np.int32)
    if sel.size:
        paths[:sel.size, 0, 0] = x[sel]
        paths[:sel.size, 0, 1] = y[sel]
    status = np.zeros(n, dtype=np.int8)
    hit = np.zeros(n, dtype=np.int32)
    steps = np.zeros(n, dtype=np.int32)
    rc = lib().oracle_trace(
        n, _p(x, _f64), _p(y, _f64), _p(vx, _f64), _p(vy, _f64), _p(qm, _f64),
        _p(ex, _f64), _p(ey, _f64), _p(v8, _u8), nx, ny,
        float(p.dx), float(p.cfl), int(p.max_steps), int(is_tapered(p)),
        _p(phi, _f64), _p(wface, _f64),
        _p(rf_ex, _f64), _p(rf_ey, _f64), _p(rf_phi, _f64),
        _p(wave, _f64), n_phase, period, dt_max, bvs, bvm, _p(clock, _f64), _p(elapsed, _f64),
        int(bool(record)), _p(endpoints, _f64), _p(slots, _i32), _p(paths, _f64),
        _p(plen, _i32), stride,
        _p(status, _i8), _p(hit, _i32), _p(steps, _i32), int(threads or default_threads()))
    if rc != 0:
        raise ValueError(f"oracle_trace rejected its arguments (code {rc})")
    return dict(x=x, y=y, vx=vx, vy=vy, status=status, hit=hit, steps=steps,
                endpoints=endpoints, selected=sel,
                paths=[paths[k, :plen[k]].copy() for k in range(sel.size)],
                clock=clock, elapsed=elapsed, period=period)


def counts_from_detail(d, spc, shape):
    """Per-species hit histograms, escapes and lost count (trench_charging_2d.py:694-702)."""
    nx, ny = shape
    spc = np.asarray(spc)
    counts = [np.bincount(d["hit"][(d["status"] == 1) & (spc == k)], minlength=nx * ny).reshape(nx, ny)
              for k in (0, 1)]
    escaped = np.bincount(spc[d["status"] == 2], minlength=2).astype(np.int64)
    lost = int(np.count_nonzero(d["status"] == 3))
    return counts[0], counts[1], escaped, lost


def trace(x, y, vx, vy, qm, spc, Ex, Ey, vac, p, barrier=None, record=None, stop=None, rf=None,
          threads=None):
    """Drop-in restatement of ``trace_cpu`` (trench_charging_2d.py:542)."""
    vac = np.asarray(vac, dtype=bool)
    n = len(x)
    if stop is not None and stop.is_set():
        # The reference loop checks the event before every step (trench_charging_2d.py:582).
        d = dict(x=np.asarray(x, float).copy(), y=np.asarray(y, float).copy(),
                 vx=np.asarray(vx, float).copy(), vy=np.asarray(vy, float).copy(),
                 status=np.full(n, 3, np.int8), hit=np.full(n, -1, np.int32),
                 steps=np.zeros(n, np.int32), endpoints=np.column_stack((x, y)).astype(float),
                 selected=selected_paths(n, p.probe_trajectories) if record is not None else None,
                 paths=None, clock=None, elapsed=None)
        if record is not None:
            d["paths"] = [np.array([[x[k], y[k]]], dtype=float) for k in d["selected"]]
            if rf is not None:
                d["clock"] = np.asarray(rf["initial_time"], float) % rf["period"]
                d["elapsed"] = np.zeros(n)
                d["period"] = rf["period"]
    else:
        d = trace_detail(x, y, vx, vy, qm, Ex, Ey, vac, p, barrier, rf, record is not None,
                         p.probe_trajectories if record is not None else 0, threads)
    out = counts_from_detail(d, spc, vac.shape)
    if record is not None:
        nx, ny = vac.shape
        cells = np.full((n, 2), -1, dtype=int)
        ab = d["status"] == 1
        cells[ab] = np.column_stack((d["hit"][ab] // ny, d["hit"][ab] % ny))
        record.update(selected=d["selected"], status=d["status"], hit_cells=cells,
                      initial_x=np.asarray(x).copy(), endpoints=d["endpoints"],
                      final_velocity=np.column_stack((d["vx"], d["vy"])), paths=d["paths"],
                      cancelled=stop is not None and stop.is_set())
        if rf is not None:
            period = rf["period"]
            record.update(launch_phase=(np.asarray(rf["initial_time"]) % period) / period * 360,
                          final_phase=d["clock"] / period * 360, flight_time=d["elapsed"])
    return out
