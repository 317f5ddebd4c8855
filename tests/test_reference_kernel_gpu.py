"""The reference's own FP64 CUDA kernel (trench_trace.cu, compiled unmodified for
sm_100a into oracle/_ref by `make -C oracle ref`) run on the B200:

* it reproduces the reference CPU tracer on the golden cases (the reference's
  own CPU/CUDA agreement, tests/test_cuda.py:49-79), and the B200 FP64 kernel
  reproduces it;
* it is the plain single-case FP64 GPU form the FP32 path is measured against.
  The timing comparison writes its numbers to $TB_REPORT_DIR/reference_kernel.json
  when that variable is set.
"""
import json
import os
import time

import numpy as np
import pytest

from conftest import load_golden
from oracle import ref_cuda

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_cuda.available(), reason="oracle/_ref/trench_trace.cubin not built")]

CASES = ["small_barrier", "small_absorb", "taper_barrier", "taper_absorb", "cfg1", "cfg2"]


def parts(g):
    return [g[k].copy() for k in ("x", "y", "vx", "vy", "qm", "spc")]


def barrier(g):
    return (g["phi"], g["wface"]) if bool(g["barrier"]) else None


@pytest.mark.parametrize("name", CASES)
def test_reference_kernel_reproduces_reference_cpu_and_b200_fp64(cuda_device, name):
    from trench_b200.tracer import B200Tracer
    g = load_golden(f"trace_{name}.npz")
    ref = ref_cuda.RefCudaTracer(~g["solid"], cuda_device)
    got = ref(*parts(g), g["Ex"], g["Ey"], ~g["solid"], g["p"], barrier(g))
    np.testing.assert_array_equal(got[0], g["cnt_i"])
    np.testing.assert_array_equal(got[1], g["cnt_e"])
    np.testing.assert_array_equal(got[2], g["escaped"])
    assert got[3] == int(g["lost"])
    mine = B200Tracer(~g["solid"], cuda_device, precision="f64")(*parts(g), g["Ex"], g["Ey"], ~g["solid"],
                                                                  g["p"], barrier(g))
    for a, b in zip(got, mine):
        np.testing.assert_array_equal(a, b)


def fresh_fields(Ex, Ey, solid, k):
    """Copies of the fields that differ in bits from every other repetition's (a solid
    cell's field, which no tracer reads through its zero vacuum weight, is offset by k), so
    no call can reuse a previous call's field upload."""
    ex = Ex.copy()
    ix, iy = np.argwhere(solid)[0]
    ex[ix, iy] += float(k)
    return ex, Ey.copy()


def timed_calls(fn, prt, Ex, Ey, solid, rest, reps, rf=None):
    """Best wall time of `reps` tracer calls (synchronised on both sides), each on fresh
    copies of the particles and fields made before its timed region; returns the last
    call's output and the time."""
    import torch
    out, ts = None, []
    for k in range(reps):
        args = [a.copy() for a in prt]
        ex, ey = fresh_fields(Ex, Ey, solid, k)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn(*args, ex, ey, *rest, **({} if rf is None else {"rf": rf}))
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    return out, min(ts)


def test_speed_against_plain_fp64_gpu_form(cuda_device):
    """Same 2^20 particles of the benchmark workload on the charged AR-8 fields: the
    reference FP64 kernel driven like the reference (per-256-step host syncs, host
    bincount) against the B200 FP32 and FP64 tracers through the same host-array call.
    The FP32 call must be at least 5x the reference kernel's."""
    import bench
    from trench_b200 import inject
    from trench_b200.tracer import B200Tracer
    g = load_golden("trace_cfg2.npz")
    p = bench.workload()
    solid = g["solid"]
    prt = inject.inject(p, p.n_per_batch, solid.shape[1], np.random.default_rng(5), ion_velocity=bench.ion_sampler(p))
    rest = (~solid, p, (g["phi"], g["wface"]))
    ref = ref_cuda.RefCudaTracer(~solid, cuda_device)
    f32 = B200Tracer(~solid, cuda_device, precision="f32")
    f64 = B200Tracer(~solid, cuda_device, precision="f64")
    timed_calls(ref, prt, g["Ex"], g["Ey"], solid, rest, 1)
    timed_calls(f32, prt, g["Ex"], g["Ey"], solid, rest, 1)
    r_ref, t_ref = timed_calls(ref, prt, g["Ex"], g["Ey"], solid, rest, 3)
    r_f32, t_f32 = timed_calls(f32, prt, g["Ex"], g["Ey"], solid, rest, 3)
    r_f64, t_f64 = timed_calls(f64, prt, g["Ex"], g["Ey"], solid, rest, 2)
    for a, b in zip(r_ref, r_f64):
        np.testing.assert_array_equal(a, b)
    n = len(prt[0])
    steps = f32.last["particle_steps"]
    report = {"particles": n, "particle_steps": steps,
              "reference_fp64_kernel_s": t_ref, "b200_f32_call_s": t_f32, "b200_f64_call_s": t_f64,
              "speedup_f32_vs_reference_kernel": t_ref / t_f32, "speedup_f64_vs_reference_kernel": t_ref / t_f64,
              "reference_launches": ref.launches}
    print(json.dumps(report))
    out = os.environ.get("TB_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "reference_kernel.json"), "w") as fh:
            json.dump(report, fh, indent=1)
    assert t_ref / t_f32 >= 5.0


def rf_of(g):
    return dict(period=float(g["rf_period"]), dt_max=float(g["rf_dt_max"]), wave=g["rf_wave"], phi=g["rf_phi"],
                Ex=g["rf_Ex"], Ey=g["rf_Ey"], initial_time=g["rf_initial_time"])


def test_reference_kernel_with_rf_clock_reproduces_reference_cpu_and_b200_fp64(cuda_device):
    """The in-flight RF clock: the reference kernel, the reference CPU tracer (fixture) and the
    B200 FP64 kernel give the same counts."""
    from trench_b200.tracer import B200Tracer
    g = load_golden("trace_rf_taper.npz")
    args = (g["Ex"], g["Ey"], ~g["solid"], g["p"], barrier(g))
    got = ref_cuda.RefCudaTracer(~g["solid"], cuda_device)(*parts(g), *args, rf=rf_of(g))
    mine = B200Tracer(~g["solid"], cuda_device, precision="f64")(*parts(g), *args, rf=rf_of(g))
    for a, b, want in zip(got, mine, (g["cnt_i"], g["cnt_e"], g["escaped"])):
        np.testing.assert_array_equal(a, want)
        np.testing.assert_array_equal(b, want)
    assert got[3] == mine[3] == int(g["lost"])


def test_circuit_rf_batch_against_the_reference_kernel(cuda_device):
    """One batch of the reference's circuit_rf benchmark run (120 x 560 grid, pulsed 5 kV,
    3000 ions + 3000 electrons at stratified phases): the reference kernel driven like the
    reference and the B200 FP64 kernel give the same counts; the B200 FP32 kernel agrees on
    >= 99.9 % of the particles' outcomes; both B200 kernels are faster than the reference
    kernel (a batch this small is bound by the step latency of its longest trajectories,
    not by throughput)."""
    import torch
    import bench
    from trench_b200 import geometry, inject
    from trench_b200.fields import compute_field, setup_fields
    from trench_b200.tracer import B200Tracer
    p, circuit, _, _ = bench.rf_cycle_workload()
    solid, mask, _, _ = geometry.build_geometry(p)
    f = setup_fields(p, solid, mask, circuit, device=cuda_device)
    ex, ey = compute_field(f["external"], ~solid, p, f["volts"]["top"])
    wface = np.where(f["cond"], 1.0, f["eps"] / (1 + f["eps"]))
    rng = np.random.default_rng(9)
    prt = inject.inject(p, p.n_per_batch, solid.shape[1], rng, ion_energy=lambda r, k: np.full(k, p.electron_temp_eV / 2))
    rf = {**f["rf"], "initial_time": np.concatenate([inject.launch_times(rng, p.n_per_batch, f["rf"]["period"])
                                                     for _ in range(2)])}
    args = (ex, ey, ~solid, p, (f["external"], wface))
    ref = ref_cuda.RefCudaTracer(~solid, cuda_device)
    f64 = B200Tracer(~solid, cuda_device, precision="f64")
    f32 = B200Tracer(~solid, cuda_device, precision="f32")

    rest = args[2:]
    r_ref, t_ref = timed_calls(ref, prt, ex, ey, solid, rest, 2, rf=rf)
    r_f64, t_f64 = timed_calls(f64, prt, ex, ey, solid, rest, 2, rf=rf)
    r_f32, t_f32 = timed_calls(f32, prt, ex, ey, solid, rest, 3, rf=rf)
    for a, b in zip(r_ref[:3], r_f64[:3]):
        np.testing.assert_array_equal(a, b)
    assert r_ref[3] == r_f64[3]
    same = (f32.last["status"] == f64.last["status"]) & (f32.last["hit"] == f64.last["hit"])
    report = {"workload": "circuit_rf benchmark run, one batch of 6000 particles", "reference_fp64_kernel_s": t_ref,
              "b200_f64_call_s": t_f64, "b200_f32_call_s": t_f32, "f32_agreement": float(same.mean()),
              "reference_launches": ref.launches}
    print(json.dumps(report))
    out = os.environ.get("TB_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "reference_kernel_rf.json"), "w") as fh:
            json.dump(report, fh, indent=1)
    assert same.mean() >= 0.999
    assert t_f32 < t_ref
    assert t_f64 < t_ref
