"""Case packs: many cases in one persistent launch give exactly the per-case results."""
from dataclasses import replace

import numpy as np
import pytest

from trench_b200 import inject
from trench_b200.batch import sweep_params

pytestmark = pytest.mark.gpu


def small_sweep():
    ps, _ = sweep_params(5, seed=3)
    # keep the setup quick: short trenches and few particles
    return [replace(p, trench_d=min(p.trench_d, 60), trench_taper_deg=min(p.trench_taper_deg, 2.0),
                    n_per_batch=1500 + 700 * i, n_batches=3) for i, p in enumerate(ps)]


@pytest.mark.parametrize("order", ["reverse", "learned", "index"])
def test_pack_equals_cases_traced_one_by_one(cuda_device, order):
    """Every claim order of the pack (the learned one through the batched ordering
    kernels and claim records) gives each case's results bit for bit."""
    from trench_b200.batch import ChargingBatch
    from trench_b200.step import ChargingCase
    ps = small_sweep()
    batch = ChargingBatch(ps, device=cuda_device, max_batches=4, claim_order=order)
    singles = [ChargingCase(p, device=cuda_device, precision="f32", max_batches=4) for p in ps]
    rngs = [np.random.default_rng(100 + i) for i in range(len(ps))]
    for _ in range(3):
        for i, (p, c) in enumerate(zip(ps, singles)):
            parts = inject.inject(p, p.n_per_batch, c.ny, rngs[i])
            batch.load(i, *parts)
            c.load(*parts)
            c.step()
        batch.step()
    batch.check()
    for b, c in zip(batch.cases, singles):
        c.check()
        np.testing.assert_array_equal(b.rho(), c.rho())
        hb, hc = b.history(), c.history()
        for k in hc:
            np.testing.assert_array_equal(hb[k], hc[k])


@pytest.mark.parametrize("order", ["reverse", "learned"])
def test_pack_graph_replay(cuda_device, order):
    import torch
    from trench_b200.batch import ChargingBatch
    ps = small_sweep()[:3]
    a = ChargingBatch(ps, device=cuda_device, max_batches=4, claim_order=order)
    b = ChargingBatch(ps, device=cuda_device, max_batches=4, claim_order=order)
    for i, p in enumerate(ps):
        parts = inject.inject(p, p.n_per_batch, a.cases[i].ny, np.random.default_rng(7 + i))
        a.load(i, *parts)
        b.load(i, *parts)
    a.step()
    a.step()
    b.capture()
    b.replay()
    b.replay()
    torch.cuda.synchronize()
    for ca, cb in zip(a.cases, b.cases):
        np.testing.assert_array_equal(ca.rho(), cb.rho())


def test_pack_with_circuit_rf_case_equals_cases_one_by_one(cuda_device):
    """A circuit_rf case (in-flight clock, FP32 basis fields) shares the persistent launch
    with DC cases and gives exactly its single-case result, the others too."""
    from conftest import load_golden
    from trench_b200.batch import ChargingBatch
    from trench_b200.step import ChargingCase
    g = load_golden("run_rf_taper.npz")
    circuit = dict(t=g["circuit_t"], uw=g["circuit_uw"], um=g["circuit_um"], up=g["circuit_up"], V1=g["circuit_V1"])
    ps = [replace(g["p"], n_per_batch=1200)] + small_sweep()[:2]
    circuits = [circuit, None, None]
    batch = ChargingBatch(ps, device=cuda_device, max_batches=4, circuits=circuits)
    singles = [ChargingCase(p, device=cuda_device, precision="f32", max_batches=4, circuit=c)
               for p, c in zip(ps, circuits)]
    rngs = [np.random.default_rng(200 + i) for i in range(len(ps))]
    for _ in range(2):
        for i, (p, c) in enumerate(zip(ps, singles)):
            parts = inject.inject(p, p.n_per_batch, c.ny, rngs[i])
            t0 = None
            if circuits[i] is not None:
                t0 = inject.launch_times(rngs[i], 2 * p.n_per_batch, c.rf["period"])
            batch.load(i, *parts, launch_times=t0)
            c.load(*parts, launch_times=t0)
            c.step()
        batch.step()
    batch.check()
    for b, c in zip(batch.cases, singles):
        c.check()
        np.testing.assert_array_equal(b.rho(), c.rho())
        np.testing.assert_array_equal(b.history()["ratio_i_bottom"], c.history()["ratio_i_bottom"])
