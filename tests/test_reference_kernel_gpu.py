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


def test_speed_against_plain_fp64_gpu_form(cuda_device):
    """Same 2^20 particles of the benchmark workload on the charged AR-8 fields:
    reference FP64 kernel driven like the reference (per-256-step host syncs, host
    bincount) against the B200 FP32 and FP64 tracers through the same call."""
    import torch
    import bench
    from trench_b200 import inject
    from trench_b200.tracer import B200Tracer
    g = load_golden("trace_cfg2.npz")
    p = bench.workload()
    solid = g["solid"]
    prt = inject.inject(p, p.n_per_batch, solid.shape[1], np.random.default_rng(5), ion_velocity=bench.ion_sampler(p))
    args = (g["Ex"], g["Ey"], ~solid, p, (g["phi"], g["wface"]))
    ref = ref_cuda.RefCudaTracer(~solid, cuda_device)
    f32 = B200Tracer(~solid, cuda_device, precision="f32")
    f64 = B200Tracer(~solid, cuda_device, precision="f64")

    def timed(fn, reps):
        out, ts = None, []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn(*(a.copy() for a in prt), *args)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return out, min(ts)

    timed(ref, 1)
    timed(f32, 1)
    r_ref, t_ref = timed(ref, 3)
    r_f32, t_f32 = timed(f32, 3)
    r_f64, t_f64 = timed(f64, 2)
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
    assert t_f32 < t_ref
