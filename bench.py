"""Benchmark of the per-batch charging step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload: AR-8 RF-charging trench (60x250 cells of 5 nm, trench 20x160 with a
2 deg taper, dielectric mask 20 cells eps_r 3 with a 5 deg taper), 2^19 ions +
2^19 electrons per batch, bimodal ion energy distribution (Gaussians at 40 and
140 eV, sigma 6 eV, equal weights), half-Gaussian angles (sigma 3 deg),
electrons Te 3 eV, sheet leakage 1e-15 S, barrier wall model.  Synthetic,
seeded inputs.  A step is one charging batch: trace -> deposit -> leakage ->
potential -> field, on the device, replayed from a CUDA graph.

value: traced particles per second over the timed steps (device-resident inputs,
L2 flushed between steps, CUDA events).  e2e: the same through the public API
with every step's batch copied from pinned host memory (HostPipeline: the copy of
batch k+1 overlaps batch k) and its history row read back, timed over all steps.  Under torchrun every rank runs its own case (weak scaling, no
collective on the data path); rank 0 prints the line.

--impl reference times the reference algorithm on the host cores (the FP64 C
restatement of the reference tracer plus the NumPy/SciPy batch update) on a
bounded sample of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from dataclasses import replace
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "traced particles/s and batches/s on 1 B200 at <=1% flux error vs plain FP64 form"
L2_FLUSH_BYTES = 256 << 20


def workload(n_per_species=1 << 19):
    from trench_b200.params import Params
    return replace(Params(), nx=60, trench_w=20, trench_d=160, floor_t=10, mask_t=20, n_vac=60,
                   trench_taper_deg=2.0, mask_taper_deg=5.0, mask_type="dielectric", mask_eps_r=3.0,
                   electron_temp_eV=3.0, bias="rf", field_mode="floating", sigma_s=1e-15,
                   n_per_batch=n_per_species, seed=1)


def ion_sampler(p):
    from trench_b200 import inject
    energy = inject.mixture_energy([(0.5, "normal", 40.0, 6.0), (0.5, "normal", 140.0, 6.0)])
    return inject.energy_angle_sampler(p, energy, inject.half_gaussian_angle(3.0))


def config(p, extra=None):
    c = {"workload": "AR-8 RF-charging trench, 60x250 cells, 2^20 particles/batch, bimodal IED 40/140 eV, "
                     "half-Gaussian IAD 3 deg, Te 3 eV, leakage 1e-15 S, barrier walls",
         "grid": [p.nx, p.floor_t + p.trench_d + p.mask_t + p.n_vac], "particles_per_batch": 2 * p.n_per_batch,
         "max_steps": p.max_steps, "cfl": p.cfl}
    if extra:
        c.update(extra)
    return c


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def reduce_max(value, device=None):
    """Max of a per-rank number over all ranks (the timing rule: the slowest rank sets the
    time); identity without a process group.  Works on NCCL (device tensor) and gloo."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_workload(p, rank):
    """Weak scaling: every rank runs its own case of the same workload (own seed)."""
    return replace(p, seed=p.seed + rank)


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


def profile_issue():
    """Warp instructions per particle-step of the FP32 tracer from the committed ncu summary."""
    try:
        d = json.loads((ROOT / "profiles" / "trace_f32_issue.json").read_text())
        return float(d["warp_instructions_per_particle_step"]), int(d["sms"]), int(d["schedulers_per_sm"])
    except Exception:
        return None


def profile_traffic():
    """DRAM bytes per particle of the FP32 tracer from the committed ncu summary, if any."""
    try:
        d = json.loads((ROOT / "profiles" / "trace_f32_traffic.json").read_text())
        return float(d["dram_bytes_per_particle"]), float(d.get("dram_bytes_per_step", 0.0))
    except Exception:
        return None


def cpu_baseline(p, sample_per_species, seconds_budget=20.0):
    """The oracle (FP64 C restatement of the reference tracer, all host threads) plus the
    oracle batch update, on a bounded sample of this workload."""
    from oracle import oracle_fields as OF
    from oracle import oracle_trace as OT
    from trench_b200 import geometry, inject
    threads = OT.default_threads()
    q = replace(p, n_per_batch=sample_per_species)
    solid, mask, _, _ = geometry.build_geometry(q)
    st = OF.BatchState(q, solid, mask)
    rng = np.random.default_rng(7)
    sampler = ion_sampler(q)
    done, t_total, batches = 0, 0.0, 0
    while t_total < seconds_budget and batches < 50:
        parts = inject.inject(q, q.n_per_batch, solid.shape[1], rng, ion_velocity=sampler)
        t0 = time.perf_counter()
        out = OT.trace(*parts, st.Ex, st.Ey, ~solid, q, st.barrier(), threads=threads)
        st.step(*out)
        t_total += time.perf_counter() - t0
        done += 2 * q.n_per_batch
        batches += 1
    return {"value": done / t_total, "unit": "particles/s", "cores": threads, "kind": "port",
            "sample": f"{batches} batches of {2 * sample_per_species} particles (same geometry and "
                      f"distributions, {sample_per_species} per species), trace + batch update, "
                      f"{t_total:.1f} s", "batches_per_s": batches / t_total}


def run_reference(args, p):
    """The reference arm: the reference algorithm on the host cores -- the oracle's FP64 C
    restatement of the reference tracer on all host threads plus the NumPy/SciPy batch
    update -- on this workload's own configuration: 2^19 ions + 2^19 electrons per batch,
    the warm-up batches charging the case as the B200 arm's warm-up does, then the timed
    batches, each a full batch.  Rank 0 only."""
    from oracle import oracle_fields as OF
    from oracle import oracle_trace as OT
    from trench_b200 import geometry, inject
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = OT.default_threads()
    solid, mask, _, _ = geometry.build_geometry(p)
    st = OF.BatchState(p, solid, mask)
    rng = np.random.default_rng(100)
    sampler = ion_sampler(p)
    times = []
    for i in range(args.warmup + args.steps):
        parts = inject.inject(p, p.n_per_batch, solid.shape[1], rng, ion_velocity=sampler)
        t0 = time.perf_counter()
        st.step(*OT.trace(*parts, st.Ex, st.Ey, ~solid, p, st.barrier(), threads=threads))
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    n = 2 * p.n_per_batch
    sec = float(np.sum(times))
    value = n * args.steps / sec
    line = {"metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * sec / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": config(p),
            "cpu_baseline": {"value": value, "unit": "particles/s", "cores": threads, "kind": "port",
                             "sample": f"{args.steps} full batches of {n} particles after {args.warmup} charging "
                                       f"batches, trace + batch update, {sec:.1f} s"},
            "batches_per_s": args.steps / sec,
            "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args, p):
    import torch
    import torch.distributed as dist
    from trench_b200 import inject
    from trench_b200.step import ChargingCase

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    n_steps = args.warmup + args.steps
    case = ChargingCase(rank_workload(p, rank), device=local, precision="f32", green="f64",
                        max_batches=2 * n_steps + 8, autotune=True)
    ny = case.ny
    sampler = ion_sampler(p)
    rng = np.random.default_rng(100 + rank)
    pool_n = min(n_steps, 6)
    host = []
    for _ in range(pool_n):
        parts = inject.inject(p, p.n_per_batch, ny, rng, ion_velocity=sampler)
        host.append([torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in parts])
    dev_pool = [[t.to(dev) for t in h] for h in host]
    n = 2 * p.n_per_batch
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    # graph with externally visible timing events around the tracer kernel
    t0e = torch.cuda.Event(enable_timing=True, external=True)
    t1e = torch.cuda.Event(enable_timing=True, external=True)
    # warm-up 1 and 2: eager batches; then the tracer settings are tuned on a loaded
    # batch of the (now charging) case, and the step is captured
    for i in range(2):
        case.load(*dev_pool[i % pool_n])
        case.step()
    case.load(*dev_pool[2 % pool_n])
    apply_tracer_setting(case, args.tracer_shape, n)
    torch.cuda.synchronize()
    case.trace_events = (t0e, t1e)
    graph_ok = True
    try:
        case.capture(n)
    except Exception as exc:  # noqa: BLE001
        graph_ok = False
        print(f"# CUDA graph capture failed, timing eager launches: {exc}", file=sys.stderr)

    def one_step(i):
        src = dev_pool[i % pool_n]
        for dst, s in zip(case.X + [case.SPC], src):
            dst[:n].copy_(s)
        if graph_ok:
            case.replay()
        else:
            case.step(n)

    for i in range(2, args.warmup):
        one_step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    clocks = Clocks(local)
    clocks.start()
    steps_before = case.batches_done()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    trace_ms = []
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")
    wall0 = time.perf_counter()
    for k in range(args.steps):
        src = dev_pool[(args.warmup + k) % pool_n]
        for dst, s in zip(case.X + [case.SPC], src):
            dst[:n].copy_(s)
        starts[k].record()
        if graph_ok:
            case.replay()
        else:
            case.step(n)
        ends[k].record()
        flush.zero_()
        ends[k].synchronize()
        trace_ms.append(t0e.elapsed_time(t1e))
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    torch.cuda.nvtx.range_pop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    total_ms = reduce_max(total_ms, dev)
    hist = case.history()
    steps_per_batch = hist["particle_steps"][steps_before:steps_before + args.steps]

    # e2e: host buffers through the public API: every step's batch is copied from pinned
    # host memory (overlapping the previous step's compute) and its history row read back
    from trench_b200.step import HostPipeline
    pipe = HostPipeline(case, n)
    # batches without qm: each particle's charge-to-mass ratio is its species' (HostPipeline)
    batches = [host[k % pool_n][:4] + host[k % pool_n][5:] for k in range(args.steps)]
    rows = torch.empty((args.steps, case.hist_cols), dtype=torch.float64).pin_memory()
    pipe.run(batches[:2], rows[:2])                      # warm the second graph
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record()
    pipe.run(batches, rows, between=flush.zero_)
    s1.record()
    s1.synchronize()
    e2e_total = s0.elapsed_time(s1)
    row = rows[0]
    # device injection: the batch is drawn on the GPU (Philox) inside the captured graph
    dinj = device_injection(case, p, args.steps)
    clk = clocks.stop()
    case.check()
    h2d = sum(t.numel() * t.element_size() for t in batches[0])
    d2h = row.numel() * row.element_size()
    e2e_total = reduce_max(e2e_total, dev)

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    acc = accuracy_measure(case, host[0]) if world == 1 else None
    fp64_gpu = fp64_gpu_baseline(case, host[0], total_ms / args.steps) if world == 1 else None
    adj = adjoint_measure() if (args.adjoint and world == 1) else None
    to_steady = steady_measure(p) if (args.steady and world == 1) else None
    sweep = large = None
    if args.configs and world == 1:
        sweep = sweep_measure(3, 3, args.cases, cpu_seconds=5.0)
        torch.cuda.empty_cache()
        large = large_measure(3, 3, cpu_seconds=5.0, tracer_reps=1)
        torch.cuda.empty_cache()

    particles = n * args.steps * world
    value = particles / (total_ms / 1000.0)
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    hbm_source = "of measured (MEASURED_PEAKS.json)" if "hbm_gbs" in peaks else "of fallback (6.65 TB/s)"
    # Tracer roofline: algorithmic bytes = 36 B per particle-step (4 bilinear corners of
    # Ex, Ey, vacuum in FP32) + 28 B per particle (SoA load + status/hit store).
    alg_bytes = [36.0 * s + 28.0 * n for s in steps_per_batch]
    achieved = float(np.mean([b / (t / 1000.0) for b, t in zip(alg_bytes, trace_ms)])) / 1e9
    smem_peak = case_smem_peak(case)
    traffic = profile_traffic()
    mean_steps = float(np.mean(steps_per_batch))
    roof = {"bound": "smem", "achieved": achieved, "peak": smem_peak, "unit": "GB/s",
            "frac": achieved / smem_peak if smem_peak else None,
            "peak_source": "measured shared-memory load bandwidth (bench microkernel)",
            "traffic": (traffic[0] * n + traffic[1] * mean_steps) if traffic else None,
            "hbm_peak_gbs": hbm, "hbm_frac_of_measured": (achieved / hbm) if hbm else None,
            "hbm_peak_source": hbm_source,
            "kernel": "trace_f32_kernel", "trace_ms_per_launch": float(np.mean(trace_ms)),
            "particle_steps_per_launch": mean_steps,
            "particle_steps_per_s": float(np.mean([s / (t / 1000.0) for s, t in zip(steps_per_batch, trace_ms)]))}
    issue = profile_issue()
    if issue and clk and clk.get("sm_mhz"):
        # the binding limit of this kernel: one warp instruction per scheduler per cycle
        per_step, sms, sched = issue
        ach = per_step * float(np.mean([s / (t / 1000.0) for s, t in zip(steps_per_batch, trace_ms)]))
        peak = sms * sched * clk["sm_mhz"] * 1e6
        roof["issue"] = {"achieved": ach, "peak": peak, "unit": "warp instructions/s", "frac": ach / peak,
                         "warp_instructions_per_particle_step": per_step,
                         "source": "profiles/trace_f32_issue.json (ncu) x live particle-steps/s; peak = "
                                   "SMs x 4 schedulers x sampled SM clock"}
    cpu = cpu_baseline(p, 1 << 15, seconds_budget=args.cpu_seconds)
    line = {"metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config(p, {"l2": "flushed between timed steps (256 MiB write)",
                                 "graph": graph_ok, "precision": "f32 tracer, f64 Green's operator, "
                                 "f64 charge/leakage/conductor", "parallelism": f"{world} independent cases",
                                 "tracer_shape": list(case.tuning.get("tracer_shape", ())),
                                 "claim_order": case.tuning.get("claim_order"),
                                 "poisson_schedule": list(case.tuning.get("poisson_schedule", ()))}),
            "batches_per_s": 1000.0 * args.steps * world / total_ms,
            "e2e": {"value": particles / (e2e_total / 1000.0), "unit": "particles/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "batches_per_s": 1000.0 * args.steps * world / e2e_total,
                    "batch": "HostPipeline.run: x, y, vx, vy (FP64) and species (int8) per particle from pinned "
                             "host memory, q/m from the species on the device; history row read back"},
            "device_injection": dinj,
            "accuracy": acc,
            "fp64_gpu_baseline": fp64_gpu,
            "sweep": sweep,
            "large": large,
            "adjoint": adj,
            "to_steady": to_steady,
            # per step: batch reset, tracer, fused charge update, Green's GEMV, field, monitors,
            # and with the learned claim order its three ordering kernels before the tracer and
            # two after it
            "gpu_launches": step_launches(case) * args.steps,
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            "wall_s": wall}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def sweep_cpu_baseline(ps, seps, seconds_budget=15.0, per_species=1 << 12):
    """The oracle (FP64 C tracer on all host threads + the FP64 batch update) on the sweep's
    cases in turn, each with a bounded sample of its own distributions: particles/s."""
    from oracle import oracle_fields as OF
    from oracle import oracle_trace as OT
    from trench_b200 import geometry, inject
    threads = OT.default_threads()
    rng = np.random.default_rng(12)
    done, t_total, cases = 0, 0.0, 0
    for p, sep in zip(ps[:16], seps[:16]):
        if t_total >= seconds_budget:
            break
        q = replace(p, n_per_batch=per_species)
        solid, mask, _, _ = geometry.build_geometry(q)
        st = OF.BatchState(q, solid, mask)
        energy = inject.mixture_energy([(0.5, "normal", 40.0, 6.0), (0.5, "normal", 40.0 + sep, 6.0)])
        sampler = inject.energy_angle_sampler(q, energy, inject.half_gaussian_angle(3.0))
        parts = inject.inject(q, q.n_per_batch, solid.shape[1], rng, ion_velocity=sampler)
        t0 = time.perf_counter()
        st.step(*OT.trace(*parts, st.Ex, st.Ey, ~solid, q, st.barrier(), threads=threads))
        t_total += time.perf_counter() - t0
        done += 2 * per_species
        cases += 1
    return {"value": done / t_total, "unit": "particles/s", "cores": threads, "kind": "port",
            "sample": f"one batch of {2 * per_species} particles on each of the first {cases} sweep cases "
                      f"(their own geometry and distributions), trace + batch update, {t_total:.1f} s"}


def sweep_measure(steps, warmup, n_cases=64, cpu_seconds=15.0, accuracy=True):
    """Batched sweep (configuration 3): n_cases uneven cases advanced together, one
    persistent tracer launch per batch for all cases, then one launch per update stage
    for all cases; the whole batch replayed from one CUDA graph.  Returns the timings,
    the case-pack tracer's roofline, the oracle CPU baseline on the first cases and the
    FP32-vs-FP64 accuracy of one case."""
    import torch
    from trench_b200 import inject
    from trench_b200.batch import ChargingBatch, sweep_params
    dev = torch.device("cuda", torch.cuda.current_device())
    ps, seps = sweep_params(n_cases, seed=0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch = ChargingBatch(ps, device=dev.index, max_batches=warmup + steps + 4)
    setup_s = time.perf_counter() - t0
    rng = np.random.default_rng(11)
    total, loaded = 0, []
    for i, (p, sep) in enumerate(zip(ps, seps)):
        energy = inject.mixture_energy([(0.5, "normal", 40.0, 6.0), (0.5, "normal", 40.0 + sep, 6.0)])
        sampler = inject.energy_angle_sampler(p, energy, inject.half_gaussian_angle(3.0))
        parts = inject.inject(p, p.n_per_batch, batch.cases[i].ny, rng, ion_velocity=sampler)
        batch.load(i, *parts)
        loaded.append(parts)
        total += 2 * p.n_per_batch
    t0e = torch.cuda.Event(enable_timing=True, external=True)
    t1e = torch.cuda.Event(enable_timing=True, external=True)
    batch.trace_events = (t0e, t1e)
    batch.step()
    torch.cuda.synchronize()
    batch.capture()
    for _ in range(warmup - 1):
        batch.replay()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    clocks = Clocks(dev.index)
    clocks.start()
    ms, trace_ms, steps_per_batch = [], [], []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.replay()
        e1.record()
        flush.zero_()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        trace_ms.append(t0e.elapsed_time(t1e))
        steps_per_batch.append(sum(c.history()["particle_steps"][-1] for c in batch.cases))
    clk = clocks.stop()
    batch.check()
    batch._graph = None
    batch.trace_events = None
    smem = case_smem_peak(batch.cases[0])
    alg = [36.0 * st + 28.0 * total for st in steps_per_batch]
    achieved = float(np.mean([b / (t / 1000.0) for b, t in zip(alg, trace_ms)])) / 1e9
    out = {"workload": f"batched sweep: {len(ps)} cases, widths 12-40, depths 40-200, tapers -3..5 deg, mask "
                       "conductive/dielectric, particles/species log-uniform 2^15-2^17, bimodal IED separation "
                       "30-150 eV", "cases": len(ps), "particles_per_batch": total, "setup_s": setup_s,
           "steps": steps, "warmup": warmup, "ms_per_step": float(np.mean(ms)),
           "value": total / (np.mean(ms) / 1000.0), "unit": "particles/s",
           "batches_per_s": 1000.0 / float(np.mean(ms)), "trace_ms_per_batch": float(np.mean(trace_ms)),
           "update_ms_per_batch": float(np.mean(ms) - np.mean(trace_ms)),
           "particle_steps_per_batch": float(np.mean(steps_per_batch)),
           "roofline": {"bound": "smem", "kernel": "trace_f32_batch_kernel", "achieved": achieved, "peak": smem,
                        "unit": "GB/s", "frac": achieved / smem if smem else None,
                        "peak_source": "measured shared-memory load bandwidth (bench microkernel)",
                        "note": "36 B per particle-step + 28 B per particle over the case-pack tracer launch"},
           "l2": "flushed between timed steps (256 MiB write)", "clocks": clk,
           # per batch: the pack's reset and tracer launches, the charge update of all cases (one launch),
           # the Green's products (one launch) and the fields (one launch), and with the learned
           # claim order its five batched ordering kernels
           "gpu_launches": (5 + (5 if batch.cases[0].tuning.get("claim_order") == "learned" else 0)) * steps,
           "cpu_baseline": sweep_cpu_baseline(ps, seps, seconds_budget=cpu_seconds)}
    if accuracy:
        # the largest case of the pack, one batch from its charged state, FP32 vs FP64
        k = int(np.argmax([p.n_per_batch for p in ps]))
        out["accuracy"] = {"case": k, **accuracy_measure(batch.cases[k], loaded[k])}
    return out


def run_sweep(args):
    """Batched sweep alone: its own contract line (configuration 3)."""
    import torch
    torch.cuda.set_device(0)
    m = sweep_measure(args.steps, args.warmup, args.cases, args.cpu_seconds)
    line = {"metric": METRIC, "value": m["value"], "unit": "particles/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": m["workload"], "cases": m["cases"], "particles_per_batch": m["particles_per_batch"],
                       "setup_s": m["setup_s"], "l2": m["l2"]},
            **{k: m[k] for k in ("batches_per_s", "particle_steps_per_batch", "trace_ms_per_batch",
                                 "update_ms_per_batch", "roofline", "cpu_baseline", "accuracy", "clocks",
                                 "gpu_launches")}}
    print(json.dumps(line), flush=True)
    return 0


def large_workload(n_per_species=1 << 23):
    """Configuration 5: 1.25 nm cells, 400 x 1400 grid, trench 40 x 800 (AR 20), floor 20,
    dielectric mask 80 cells (eps_r 3), 500 vacuum rows, Te 3 eV, leakage 1e-15 S.
    max_steps 12000: crossing 1400 rows at CFL 0.35 takes more than 4000 steps, so the
    default 3000 would stop most ions short of the floor."""
    from trench_b200.params import Params
    return replace(Params(), dx=1.25e-9, nx=400, trench_w=40, trench_d=800, floor_t=20, mask_t=80, n_vac=500,
                   mask_type="dielectric", mask_eps_r=3.0, electron_temp_eV=3.0, bias="dc", field_mode="floating",
                   sigma_s=1e-15, max_steps=12000, n_per_batch=n_per_species, seed=5)


def large_tables():
    """Pulsed-bias IED: 0.1 N(150 eV, 3 eV) + 0.9 U[5, 30] eV + 0.2 exponential tail (scale
    15 eV), weights renormalised to sum 1, tabulated over 0-300 eV in 2048 bins; IAD
    half-Gaussian sigma 6 deg over 0-36 deg."""
    from trench_b200 import inject
    w = np.array([0.1, 0.9, 0.2]) / 1.2

    def pdf(e):
        g = np.exp(-0.5 * ((e - 150.0) / 3.0) ** 2) / (3.0 * np.sqrt(2 * np.pi))
        u = np.where((e >= 5.0) & (e <= 30.0), 1.0 / 25.0, 0.0)
        x = np.exp(-e / 15.0) / 15.0
        return w[0] * g + w[1] * u + w[2] * x
    et = inject.table_from_pdf(pdf, 0.0, 300.0, bins=2048)
    at = inject.table_from_pdf(inject.half_gaussian_pdf(np.radians(6.0)), 0.0, np.radians(36.0))
    return et, at


def large_cpu_baseline(case, p, sample_per_species=1 << 11, seconds_budget=10.0):
    """The oracle's FP64 C tracer (all host threads) on bounded samples of the large
    workload, drawn on the host from the same distributions, through the case's current
    fields.  Trace only: the oracle's per-batch update needs the sparse-LU factorisation
    of the 560,000-cell operator (10.5 s) and a leakage set-up over a dense 560,000 x 2,160
    right-hand side, which are not run here."""
    from oracle import oracle_trace as OT
    from trench_b200 import inject
    threads = OT.default_threads()
    q = replace(p, n_per_batch=sample_per_species)
    energy = inject.mixture_energy([(0.1, "normal", 150.0, 3.0), (0.9, "uniform", 5.0, 30.0), (0.2, "exp", 15.0, 0)])
    sampler = inject.energy_angle_sampler(q, energy, inject.half_gaussian_angle(6.0))
    ex, ey = case.fields()
    phi = case.full_potential()
    wface = case.t_wface.cpu().numpy().reshape(case.nx, case.ny)
    rng = np.random.default_rng(17)
    done, t_total, batches = 0, 0.0, 0
    while t_total < seconds_budget and batches < 20:
        parts = inject.inject(q, q.n_per_batch, case.ny, rng, ion_velocity=sampler)
        t0 = time.perf_counter()
        OT.trace(*parts, ex, ey, ~case.solid, q, (phi, wface), threads=threads)
        t_total += time.perf_counter() - t0
        done += 2 * q.n_per_batch
        batches += 1
    return {"value": done / t_total, "unit": "particles/s", "cores": threads, "kind": "port",
            "sample": f"{batches} batches of {2 * sample_per_species} particles through the case's fields, trace "
                      f"only (the 560,000-cell LU set-up is not run), {t_total:.1f} s"}


def large_measure(steps, warmup, n_per_species=1 << 23, tracer_shape="auto", cpu_seconds=10.0, accuracy=True,
                  tracer_reps=3):
    """Configuration 5 on one GPU: 2^23 ions + 2^23 electrons per batch drawn on the device
    (Philox, tabulated IED/IAD) and traced through the 400 x 1400 grid, whose packed field
    (4.5 MB) is read through L2; one batch = inject + trace + deposit + leakage + potential +
    field, replayed from a CUDA graph."""
    import ctypes
    import torch
    from trench_b200 import _capi, inject
    from trench_b200.step import ChargingCase
    p = large_workload(n_per_species)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    case = ChargingCase(p, precision="f32", green="f64", max_batches=warmup + steps + 16, autotune=True)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    et, at = large_tables()
    inj = inject.DeviceInjector(case, seed=2025, energy_table=et, angle_table=at)
    inj(batch=10 ** 6)
    n = 2 * p.n_per_batch
    apply_tracer_setting(case, tracer_shape, n, reps=tracer_reps)
    t0e = torch.cuda.Event(enable_timing=True, external=True)
    t1e = torch.cuda.Event(enable_timing=True, external=True)
    case.trace_events = (t0e, t1e)
    side = torch.cuda.Stream(case.dev)
    side.wait_stream(torch.cuda.current_stream(case.dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            inj()
            case.step(n)
    torch.cuda.current_stream(case.dev).wait_stream(side)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=case.dev)
    for _ in range(warmup):
        g.replay()
    torch.cuda.synchronize()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    before = case.batches_done()
    ms, trace_ms = [], []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        flush.zero_()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        trace_ms.append(t0e.elapsed_time(t1e))
    clk = clocks.stop()
    case.check()
    del g
    case.trace_events = None
    h = case.history()
    st = h["particle_steps"][before:before + steps]
    total = float(sum(ms))
    alg = [36.0 * x + 28.0 * n for x in st]
    achieved = float(np.mean([b / (t / 1000.0) for b, t in zip(alg, trace_ms)])) / 1e9
    field_bytes = (case.nx + 2) * (case.ny + 2) * 8
    l2 = ctypes.c_double()
    l2_ok = _capi.lib().tb_bench_l2_gather(case.ctx.handle, field_bytes, ctypes.byref(l2)) == 0
    out = {"workload": "large fine-grid case: 1.25 nm cells, 400x1400 grid, trench 40x800 (AR 20), dielectric mask "
                       "80 cells, pulsed-bias IED 0.1 N(150,3) + 0.9 U[5,30] + 0.2 exp(15 eV) renormalised, IAD "
                       "half-Gaussian 6 deg, 2^24 particles/batch, max_steps 12000, drawn on the device",
           "grid": [case.nx, case.ny], "particles_per_batch": n, "surface_cells": case.m,
           "green_rows": int(len(case.rows)), "setup_s": setup_s, "steps": steps, "warmup": warmup,
           "ms_per_step": total / steps, "value": n * steps / (total / 1000.0), "unit": "particles/s",
           "batches_per_s": 1000.0 * steps / total, "trace_ms_per_batch": float(np.mean(trace_ms)),
           "particle_steps_per_batch": float(np.mean(st)),
           "particle_steps_per_s": float(np.mean([x / (t / 1000.0) for x, t in zip(st, trace_ms)])),
           "lost_fraction": float(np.mean(h["lost"][before:before + steps])),
           "ratio_i_bottom": float(np.mean(h["ratio_i_bottom"][before:before + steps])),
           "tracer_shape": list(case.tuning.get("tracer_shape", ())), "claim_order": case.tuning.get("claim_order"),
           "roofline": {"bound": "l2", "kernel": "trace_f32_kernel (global-memory field)", "achieved": achieved,
                        "peak": l2.value if l2_ok else None, "unit": "GB/s",
                        "frac": achieved / l2.value if l2_ok and l2.value > 0 else None,
                        "peak_source": f"measured random 32-byte sector gathers from an L2-resident "
                                       f"{field_bytes / 2**20:.1f} MiB buffer (bench microkernel)",
                        "note": "36 B per particle-step + 28 B per particle over the tracer launch; a lane reuses "
                                "its four corners while it stays in one cell quad, and two of them share a "
                                "sector, so fewer sectors are fetched than the bytes counted"},
           "l2": "flushed between timed steps (256 MiB write)", "clocks": clk,
           # per step: injection, batch reset, tracer, deposit, leakage GEMV, finish (m > 1024:
           # unfused charge update), Green's GEMV, field, monitors (+ 5 with the learned order)
           "gpu_launches": (9 + (5 if case.tuning.get("claim_order") == "learned" else 0)) * steps,
           "cpu_baseline": large_cpu_baseline(case, p, seconds_budget=cpu_seconds)}
    if accuracy:
        inj()
        torch.cuda.synchronize()
        batch = [t[:n].cpu().numpy() for t in case.X + [case.SPC]]
        out["accuracy"] = accuracy_measure(case, batch)
    return out


def run_large(args):
    """Configuration 5 alone: its own contract line."""
    m = large_measure(args.steps, args.warmup, args.particles if args.particles != 1 << 19 else 1 << 23,
                      args.tracer_shape, args.cpu_seconds)
    line = {"metric": METRIC, "value": m["value"], "unit": "particles/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {k: m[k] for k in ("workload", "grid", "particles_per_batch", "surface_cells", "green_rows",
                                         "l2", "tracer_shape", "claim_order")},
            **{k: m[k] for k in ("batches_per_s", "setup_s", "particle_steps_per_batch", "particle_steps_per_s",
                                 "trace_ms_per_batch", "lost_fraction", "ratio_i_bottom", "roofline",
                                 "cpu_baseline", "accuracy", "clocks", "gpu_launches")},
            "e2e": None}
    print(json.dumps(line), flush=True)
    return 0


def rf_cycle_workload():
    """The reference's own circuit_rf benchmark run (its docs/rf_cycle_validation.json):
    5 nm cells, 120 x 560 grid, trench 80 x 400, conductive mask 60 cells, pillar sides,
    pulsed 5 kV bias at 400 kHz (duty 0.2, rise 10 ns), 3000 ions + 3000 electrons per
    batch, max_steps 10000, until_steady with at most 3000 batches.  The circuit waveform
    over one period comes from the reference's circuit model, run where the reference
    is available (tests/golden/make_circuit_rf_cycle.py); the charging step reads it.
    Returns (params, circuit, reference batches, reference seconds)."""
    from trench_b200.params import Params
    g = np.load(ROOT / "tests" / "golden" / "circuit_rf_cycle.npz")
    base = Params()
    p = replace(base, **{k: v for k, v in json.loads(str(g["params"])).items() if hasattr(base, k)})
    circuit = {k: np.asarray(g[k]) for k in ("t", "uw", "um", "up", "V1")}
    return p, circuit, int(g["reference_batches"]), float(g["reference_seconds"])


def run_rf_cycle(args):
    """The circuit_rf run of rf_cycle_workload on one GPU, whole job: batches/s with every
    batch drawn on the device (Philox; ions at Te/2, stratified launch phases) and replayed
    from one CUDA graph with the FP32 tracer (value); the same run through the public
    run() with host injection, setup included (e2e, the measure of the reference's
    published 222.6 s); and the FP64 tracer on the device-drawn batches for comparison."""
    import torch
    from trench_b200 import inject
    from trench_b200.step import ChargingCase
    p, circuit, ref_batches, ref_seconds = rf_cycle_workload()
    if args.rf_batches:
        # a shorter run (profiling): the batch cap of every leg
        p = replace(p, max_batches=min(p.max_batches, args.rf_batches))
    published = ref_batches / ref_seconds
    n = 2 * p.n_per_batch

    def device_run(precision, max_batches, seed):
        q = replace(p, max_batches=max_batches)
        case = ChargingCase(q, precision=precision, green="f64", circuit=circuit)
        inj = inject.DeviceInjector(case, seed=seed)
        inj(batch=10 ** 6)
        if precision == "f32":
            apply_tracer_setting(case, args.tracer_shape, n)
        torch.cuda.synchronize()
        clocks = Clocks(torch.cuda.current_device())
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = case.run(injector=inj)
        e1.record()
        e1.synchronize()
        clk = clocks.stop()
        nb = len(res["hist"]["t"])
        return case, res, nb, e0.elapsed_time(e1) / 1000.0, clk

    case, res, nb, sec, clk = device_run("f32", p.max_batches, 41)
    h = res["hist"]
    tail = slice(max(nb - 10, 0), nb)
    bottom = [k for k in h if k.startswith("bottom")]
    f64_case, _, nb64, sec64, _ = device_run("f64", min(300, p.max_batches), 43)
    del f64_case

    # e2e: the public run() with host injection, construction included
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hcase = ChargingCase(p, precision="f32", green="f64", circuit=circuit)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    hres = hcase.run(rng=np.random.default_rng(p.seed))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    hb = len(hres["hist"]["t"])
    W = int(p.steady_window)
    checks = hb // W
    d2h = sum(k * W * 8 * (hcase.hist_cols + len(hcase.monitor_names)) for k in range(1, checks + 1))
    line = {"metric": "charging batches/s of the circuit_rf run (reference rf_cycle_validation configuration)",
            "value": nb / sec, "unit": "batches/s", "n_gpus": 1, "steps": nb, "warmup": 1,
            "ms_per_step": 1000.0 * sec / nb, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": (nb / sec) / published, "dtype": "f32",
            "data": "synthetic particles; circuit waveform from the reference's circuit model "
                    "(tests/golden/circuit_rf_cycle.npz)",
            "config": {"workload": "circuit_rf run: 5 nm cells, 120x560 grid, trench 80x400, conductive mask 60, "
                                   "pillar sides, pulsed 5 kV at 400 kHz, 3000 ions + 3000 electrons per batch, "
                                   "max_steps 10000, until_steady (window 30, hold 2, at most 3000 batches)",
                       "grid": [case.nx, case.ny], "particles_per_batch": n, "surface_cells": case.m,
                       "rf_dt_max_s": case.rf["dt_max"], "l2": "not flushed (whole-job run)",
                       "tracer_shape": list(case.tuning.get("tracer_shape", ())),
                       "claim_order": case.tuning.get("claim_order")},
            "batches": nb, "seconds": sec, "converged": bool(res["converged"]),
            "particles_per_s": nb * n / sec,
            "lost_fraction_last_10": float(np.mean(h["lost"][tail])),
            "ratio_i_bottom_last_10": float(np.mean(h["ratio_i_bottom"][tail])),
            "bottom_potential_last_10_V": {k: float(np.mean(h[k][tail])) for k in bottom},
            "f64_tracer": {"batches": nb64, "seconds": sec64, "batches_per_s": nb64 / sec64,
                           "f32_speedup": (nb / sec) / (nb64 / sec64)},
            "published": {"batches_per_s": published, "batches": ref_batches, "seconds": ref_seconds,
                          "hardware": "RTX 5070 Ti, reference CUDA FP64 tracer, setup included"},
            "e2e": {"value": hb / wall, "unit": "batches/s", "batches": hb, "seconds": wall, "setup_s": setup_s,
                    "loop_batches_per_s": hb / (wall - setup_s), "vs_published": (hb / wall) / published,
                    "h2d_bytes_per_step": n * (5 * 8 + 1 + 16), "d2h_bytes_per_step": d2h // max(hb, 1),
                    "note": "ChargingCase construction + run(rng) with host injection (NumPy PCG64) each batch"},
            "clocks": clk,
            # per batch: injection, batch reset, tracer, deposit, leakage GEMV, finish, Green's GEMV,
            # field, monitors
            "gpu_launches": 9 * nb}
    print(json.dumps(line), flush=True)
    return 0


def standard_workload():
    """The reference's own CUDA benchmark run (its benchmark_cuda.py, recorded in its
    docs/cuda_benchmark.json): the standard geometry (5 nm cells, 60 x 200 grid, trench
    20 x 80, conductive floating mask 60 cells), DC bias, ions 100 eV with a 0.5 eV
    lateral temperature, Te 3 eV, leakage 1e-15 S, 3000 ions + 3000 electrons per batch,
    20 batches, seed 1.  Published: CPU 6.045 s, CUDA FP64 0.526 s (median of 3,
    set-up of the Poisson and leakage operators included, warm-up and plotting excluded)."""
    from trench_b200.params import Params
    return replace(Params(), dx=5e-9, nx=60, trench_w=20, trench_d=80, floor_t=10, n_vac=50, mask_t=60,
                   mask_type="conductor", field_mode="floating", ion_energy_eV=100.0, ion_temp_eV=0.5,
                   electron_temp_eV=3.0, bias="dc", sigma_s=1e-15, n_batches=20, n_per_batch=3000,
                   dt_batch=1e-4, cfl=0.35, max_steps=3000, wall_model="barrier", seed=1)


def run_standard(args):
    """The standard-geometry run of standard_workload, timed like the reference's
    benchmark: ChargingCase construction + run() of 20 batches with host injection,
    median of 3 after one warm-up run; the oracle's CPU form of the same job beside it."""
    import torch
    from oracle import oracle_fields as OF
    from oracle import oracle_trace as OT
    from trench_b200 import geometry, inject
    from trench_b200.step import ChargingCase
    p = standard_workload()
    published_cuda, published_cpu = 0.52582550002262, 6.0445344999898225
    times, setups, res = [], [], None
    clocks = Clocks(torch.cuda.current_device())
    for rep in range(4):
        torch.cuda.synchronize()
        if rep == 1:
            clocks.start()
        t0 = time.perf_counter()
        case = ChargingCase(p, precision="f32", green="f64")
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        res = case.run(rng=np.random.default_rng(p.seed))
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        if rep:
            times.append(t2 - t0)
            setups.append(t1 - t0)
        del case
    clk = clocks.stop()
    sec = float(np.median(times))
    # the oracle's CPU form of the same job: operator set-up, host injection, FP64 C tracer on
    # all host threads and the FP64 batch update
    threads = OT.default_threads()
    t0 = time.perf_counter()
    solid, mask, _, _ = geometry.build_geometry(p)
    st = OF.BatchState(p, solid, mask)
    rng = np.random.default_rng(p.seed)
    for _ in range(p.n_batches):
        parts = inject.inject(p, p.n_per_batch, solid.shape[1], rng)
        st.step(*OT.trace(*parts, st.Ex, st.Ey, ~solid, p, st.barrier(), threads=threads))
    cpu_s = time.perf_counter() - t0
    h = res["hist"]
    n = 2 * p.n_per_batch
    line = {"metric": "seconds of the reference's CUDA benchmark run (standard geometry, DC, 20 batches)",
            "value": sec, "unit": "s", "n_gpus": 1, "steps": p.n_batches, "warmup": 1,
            "ms_per_step": 1000.0 * sec / p.n_batches, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": sec / published_cuda, "dtype": "f32", "data": "synthetic (seeded host injection)",
            "config": {"workload": "standard geometry: 5 nm cells, 60x200 grid, trench 20x80, floating conductive "
                                   "mask 60, DC 100 eV ions (0.5 eV lateral), Te 3 eV, sigma_s 1e-15, "
                                   "3000 ions + 3000 electrons per batch, 20 batches",
                       "grid": list(solid.shape), "particles_per_batch": n, "timing": "construction + run(), "
                       "median of 3 after a warm-up run", "l2": "not flushed (whole-job run)"},
            "setup_s": float(np.median(setups)), "batches_per_s": p.n_batches / sec,
            "particles_per_s": n * p.n_batches / sec,
            "published": {"cuda_s": published_cuda, "cpu_s": published_cpu,
                          "hardware": "RTX 5070 Ti (CUDA FP64 tracer, CPU LU and leakage); CPU model not stated"},
            "speedup_vs_published_cuda": published_cuda / sec,
            "ratio_i_bottom_mean": float(np.mean(h["ratio_i_bottom"])),
            "cpu_baseline": {"value": cpu_s, "unit": "s", "cores": threads, "kind": "port",
                             "sample": "the whole job: operator set-up, 20 batches of 6000 particles"},
            "e2e": {"value": sec, "unit": "s", "h2d_bytes_per_step": n * (5 * 8 + 1),
                    "d2h_bytes_per_step": 0, "note": "the value is already end to end: host injection, "
                    "construction and result read-back inside the timed region"},
            "clocks": clk, "gpu_launches": None}
    print(json.dumps(line), flush=True)
    return 0


def step_launches(case):
    """This library's kernels in one device batch step of a ChargingCase with the fused
    charge update: batch reset, tracer, charge, Green's GEMV, field, monitors, plus the
    learned claim order's five ordering kernels."""
    return 6 + (5 if case.tuning.get("claim_order") == "learned" else 0)


def apply_tracer_setting(case, setting, n, reps=3):
    """'auto': the autotuner times the launch shapes and claim orders on the loaded batch;
    otherwise '<threads>x<ctas per SM>' with an optional '-reverse' claim order."""
    from trench_b200 import _capi
    if setting == "auto":
        case.autotune_tracer(n, reps=reps)
        return
    shape, _, order = setting.partition("-")
    t, c = (int(v) for v in shape.split("x"))
    L = _capi.lib()
    case.ctx.check(L.tb_set_tuning(case.ctx.handle, t, c))
    from trench_b200.step import CLAIM_ORDERS
    code = CLAIM_ORDERS.index(order) if order else 0
    case.set_claim_order(code)
    case.tuning["tracer_shape"] = (t, c)
    case.tuning["claim_order"] = CLAIM_ORDERS[code]


def device_injection(case, p, steps):
    """Particles/s when each batch is also injected on the device (tb_inject inside the
    captured graph: bimodal IED and half-Gaussian IAD tables, Maxwellian electrons)."""
    import torch
    from trench_b200 import inject
    et = inject.table_from_pdf(inject.bimodal_gaussian_pdf(40.0, 6.0, 140.0, 6.0), 0.0, 200.0)
    at = inject.table_from_pdf(inject.half_gaussian_pdf(np.radians(3.0)), 0.0, np.radians(18.0))
    inj = inject.DeviceInjector(case, seed=2024, energy_table=et, angle_table=at)
    n = 2 * p.n_per_batch
    side = torch.cuda.Stream(case.dev)
    side.wait_stream(torch.cuda.current_stream(case.dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            inj()
            case.step(n)
    torch.cuda.current_stream(case.dev).wait_stream(side)
    g.replay()
    torch.cuda.synchronize()
    ms = []
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=case.dev)
    row = torch.empty(case.hist_cols, dtype=torch.float64).pin_memory()
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        row.copy_(case.hist[min(case.batches_done() - 1, case.max_batches - 1)], non_blocking=True)
        e1.record()
        flush.zero_()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    del g
    return {"value": n / (float(np.mean(ms)) / 1000.0), "unit": "particles/s", "ms_per_step": float(np.mean(ms)),
            "h2d_bytes_per_step": 0, "d2h_bytes_per_step": row.numel() * row.element_size(),
            "note": "inject (Philox, tabulated IED/IAD) + batch step replayed from one CUDA graph; "
                    "history row read back each step"}


def accuracy_measure(case, batch):
    """The FP32 tracer against the FP64 one on one batch of the workload, from the charged
    state the bench reached (ChargingCase.compare_precisions: same particles, same charge,
    each followed by the same update)."""
    out = case.compare_precisions([t.numpy() if hasattr(t, "numpy") else t for t in batch])
    out["note"] = ("one batch of the workload from the charged state, FP32 vs FP64 tracer, same particles and "
                   "charge; bars: hit agreement >= 0.999, flux error <= 1 %, potential <= 1e-3 V")
    return out


def fp64_gpu_baseline(case, batch, step_ms, reps=3):
    """The plain single-case FP64 GPU form beside this backend, on this workload's batch
    and the charge the bench reached: the reference's own kernel (trench_trace.cu, built
    from its source for sm_100a into oracle/_ref) driven the way its host wrapper drives
    it (trench_cuda.py:100-121: particles packed and copied per call, 128-thread blocks,
    256-step launches with a host synchronisation after each, host bincount), timed
    against B200Tracer's call with the same host arrays (FP32 tracer) and against the
    device batch step.  Every call gets fresh copies of the particles and of the fields
    (bits changed in one solid cell, which no tracer reads), made outside its timing."""
    import torch
    from oracle import ref_cuda
    from trench_b200.tracer import B200Tracer
    if not ref_cuda.available():
        return {"unavailable": "oracle/_ref/trench_trace.cubin is not built (the reference tree was absent at build)"}
    ex, ey = case.fields()
    phi = case.full_potential()
    wface = case.t_wface.cpu().numpy().reshape(case.nx, case.ny)
    vac = ~case.solid
    prt = [np.array(t.numpy() if hasattr(t, "numpy") else t) for t in batch]
    ix, iy = np.argwhere(case.solid)[0]
    barrier = (phi, wface) if case.p.wall_model == "barrier" else None

    def timed(fn, k):
        best = float("inf")
        out = None
        for r in range(k):
            args = [a.copy() for a in prt]
            exr = ex.copy()
            exr[ix, iy] += float(r + 1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn(*args, exr, ey.copy(), vac, case.p, barrier)
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - t0)
        return out, 1000.0 * best

    ref = ref_cuda.RefCudaTracer(vac, case.dev.index)
    call = B200Tracer(vac, case.dev.index, precision="f32")
    timed(ref, 1)
    timed(call, 1)
    ref.launches = 0
    ref_reps = max(reps - 1, 1)
    r_ref, ref_ms = timed(ref, ref_reps)
    r_call, call_ms = timed(call, reps)
    n = len(prt[0])
    return {"workload": "one batch of this workload (2^20 particles) from the charged state the bench reached",
            "kind": "the reference's trench_trace.cu compiled unmodified for sm_100a, driven like trench_cuda.py",
            "reference_kernel_ms": ref_ms, "reference_launches_per_call": ref.launches / ref_reps,
            "b200_call_ms": call_ms, "b200_step_ms": step_ms,
            "vs_fp64_gpu_call": ref_ms / call_ms, "vs_fp64_gpu_step": ref_ms / step_ms,
            "reference_particles_per_s": n / (ref_ms / 1000.0),
            "absorbed": {"reference": int(r_ref[0].sum() + r_ref[1].sum()),
                         "b200_f32": int(r_call[0].sum() + r_call[1].sum())},
            "note": "call = B200Tracer.__call__ with host NumPy arrays (H2D copies, field pack, trace, counts back); "
                    "step = the device-resident batch step (trace + deposit + leakage + potential + field)"}


def steady_measure(p):
    """The AR-8 workload run to steady charge (configuration 2: until_steady, at most
    3000 batches, the reference's default window 30 and hold 2), each batch drawn on the
    device and replayed from a CUDA graph; the steady-state check reads the history back
    every window."""
    import time
    import torch
    from trench_b200 import inject
    from trench_b200.step import ChargingCase
    q = replace(p, until_steady=True, max_batches=3000, seed=p.seed + 7)
    case = ChargingCase(q, precision="f32", green="f64")
    et = inject.table_from_pdf(inject.bimodal_gaussian_pdf(40.0, 6.0, 140.0, 6.0), 0.0, 200.0)
    at = inject.table_from_pdf(inject.half_gaussian_pdf(np.radians(3.0)), 0.0, np.radians(18.0))
    inj = inject.DeviceInjector(case, seed=31, energy_table=et, angle_table=at)
    inj(batch=10 ** 6)
    case.autotune_tracer(2 * q.n_per_batch, reps=2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = case.run(injector=inj)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    nb = len(res["hist"]["t"])
    return {"workload": "AR-8 RF-charging trench, 2^20 particles per batch drawn on the device, until_steady "
                        "(window 30, hold 2, at most 3000 batches)",
            "converged": bool(res["converged"]), "batches": nb, "seconds": wall, "batches_per_s": nb / wall,
            "particles_per_s": nb * 2 * q.n_per_batch / wall,
            "tracer_shape": list(case.tuning.get("tracer_shape", ())), "claim_order": case.tuning.get("claim_order"),
            "steady_potentials_V": {k: round(v, 3) for k, v in res["steady"].items()}}


def adjoint_measure():
    """The adjoint on the AR-5 sensitivity workload (2^20 ions + 2^20 electrons per batch,
    50 batches, 64-bin IED, 32-bin IAD): recording time of the forward run (with 32
    field-feedback modes measured every batch), backward time of each objective, and the
    directional derivative along +-10% on the 140 eV peak's bins against central
    differences of the full charging chain on the same Philox draws."""
    import time
    import torch
    from trench_b200 import adjoint, inject
    from trench_b200.step import ChargingCase
    p, eE, wE, eA, wA = adjoint.adjoint_workload()
    B = p.n_batches
    case = ChargingCase(p, precision="f32", max_batches=B)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = adjoint.AdjointRecorder(case, eE, wE, eA, wA, seed=21).run(B)
    torch.cuda.synchronize()
    record_s = time.perf_counter() - t0
    cE = 0.5 * (eE[1:] + eE[:-1])
    vE = np.where(np.abs(cE - 140) < 15, 1.0, 0.0)
    out = {"workload": "AR-5 trench 20x100 cells (60x180 grid), floating conductive mask; 64-bin IED 0-300 eV, "
                       "32-bin IAD 0-10 deg; 2^20 ions + 2^20 electrons per batch; 50 batches; "
                       "histories checkpointed every 10 batches; 32 feedback modes measured every batch",
           "record_s": record_s, "record_particles_per_s": 2 * p.n_per_batch * B / record_s}
    f64 = torch.float64
    for name in ("phi_bottom", "ratio_i_bottom"):
        for fb in (True, False):
            gE = torch.tensor(wE, dtype=f64, device=case.dev, requires_grad=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            o = adjoint.objectives(hist, gE, None, feedback=fb)
            J = o[name] if name == "phi_bottom" else o[name][-1]
            J.backward()
            torch.cuda.synchronize()
            key = name + ("" if fb else "_frozen")
            out[f"backward_s_{key}"] = time.perf_counter() - t0
            out[f"d_{key}"] = float(np.dot(gE.grad.cpu().numpy(), wE * vE))

    def chain(w, seed=21):
        c = ChargingCase(p, precision="f32", max_batches=B)
        inj = inject.DeviceInjector(c, seed, energy_table=inject.histogram_table(eE, w),
                                    angle_table=inject.histogram_table(eA, wA))
        for _ in range(B):
            inj()
            c.step()
        h = c.history()
        return np.array([h["bottom center"][-1], h["ratio_i_bottom"][-1]])

    # the chain's derivative over 4 seeds (common random numbers within each): Richardson
    # extrapolation of central differences at h = 0.1 and 0.05 (the chain is nonlinear in
    # the weights; a central difference alone is biased by O(h^2)); the mean is the
    # comparison, the standard error the noise floor under it
    cen = lambda h, s: (chain(wE * (1 + h * vE), s) - chain(wE * (1 - h * vE), s)) / (2 * h)
    fds = np.array([(4 * cen(0.05, s) - cen(0.1, s)) / 3 for s in (21, 22, 23, 24)])
    fd, fd_se = fds.mean(axis=0), fds.std(axis=0, ddof=1) / np.sqrt(len(fds))
    out["chain_fd"] = {"phi_bottom": float(fd[0]), "ratio_i_bottom": float(fd[1]),
                       "rel_se_phi_bottom": float(fd_se[0] / abs(fd[0])),
                       "rel_se_ratio_i_bottom": float(fd_se[1] / abs(fd[1])), "seeds": 4,
                       "direction": "bins within 15 eV of 140 eV scaled by 1 +- h, Richardson of h = 0.1 and 0.05, "
                                    "common random numbers per seed"}
    for key, ref in (("phi_bottom", fd[0]), ("ratio_i_bottom", fd[1])):
        out[f"rel_err_{key}"] = abs(out[f"d_{key}"] - ref) / abs(ref)
        out[f"rel_err_{key}_frozen"] = abs(out[f"d_{key}_frozen"] - ref) / abs(ref)
    return out


def case_smem_peak(case):
    """Shared-memory load bandwidth measured on this GPU (GB/s)."""
    import ctypes
    from trench_b200 import _capi
    out = ctypes.c_double()
    code = _capi.lib().tb_bench_smem(case.ctx.handle, ctypes.byref(out))
    return out.value if code == 0 else None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--particles", type=int, default=1 << 19, help="particles per species per batch")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU-baseline sample duration")
    ap.add_argument("--workload", default="ar8", choices=["ar8", "sweep", "large", "rf_cycle", "standard"],
                    help="ar8: the AR-8 RF-charging case (default); sweep: many uneven cases per launch; "
                         "large: the 400x1400 fine-grid case with 2^24 particles per batch; rf_cycle: the "
                         "reference's circuit_rf benchmark run; standard: the reference's CUDA benchmark run")
    ap.add_argument("--cases", type=int, default=64, help="cases of the sweep workload")
    ap.add_argument("--rf-batches", type=int, default=0,
                    help="rf_cycle workload: cap every leg at this many batches (0: the full 3000)")
    ap.add_argument("--tracer-shape", default="auto",
                    help="auto (autotuned) or <threads>x<CTAs per SM>[-reverse|-learned], e.g. 1024x1-reverse")
    ap.add_argument("--no-steady", dest="steady", action="store_false",
                    help="skip the run to steady charge (AR-8 workload, 1 GPU only)")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false",
                    help="skip the adjoint measurement (AR-5 sensitivity workload, 1 GPU only)")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="skip the sweep and large-grid blocks of the default line (1 GPU only)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.workload == "sweep":
        return run_sweep(args)
    if args.workload == "large":
        return run_large(args)
    if args.workload == "rf_cycle":
        return run_rf_cycle(args)
    if args.workload == "standard":
        return run_standard(args)
    p = workload(args.particles)
    if args.impl == "reference":
        return run_reference(args, p)
    return run_b200(args, p)


if __name__ == "__main__":
    sys.exit(main())
