"""ChargingBatch: many independent trench cases advanced together.

All cases' particles are traced by one persistent launch (``tb_pack_trace``: CTAs
move between cases by remaining work, so uneven cases share every SM); the
charge, leakage, conductor, potential and field updates of all cases follow as one
launch per stage (``tb_pack_step``), and a whole batch of all cases can be
captured as one CUDA graph.  The reference runs
such a sweep as one ``run()`` per case (trench_charging_2d.py:1045).

``sweep_params`` draws the sweep workload of uneven cases (widths, depths,
tapers, mask types and particle counts).
"""
import ctypes

import numpy as np
import torch

from . import _capi, geometry
from .params import Params
from .step import CLAIM_ORDERS, ChargingCase


def sweep_params(n_cases, seed=0, base=None):
    """Cases with trench width U[12,40] cells, depth U[40,200], sidewall taper
    U[-3,5] deg, conductive or dielectric mask (equal odds), nx = width + 40,
    particles per species log-uniform in [2^15, 2^17].  Draws that close the
    opening are redrawn.  Returns (params list, per-case ion peak separations in eV)."""
    from dataclasses import replace
    rng = np.random.default_rng(seed)
    base = base or Params()
    out, seps = [], []
    while len(out) < n_cases:
        w = int(rng.integers(12, 41))
        d = int(rng.integers(40, 201))
        taper = float(rng.uniform(-3.0, 5.0))
        mask = "conductor" if rng.random() < 0.5 else "dielectric"
        n = int(round(2 ** rng.uniform(15, 17)))
        sep = float(rng.uniform(30.0, 150.0))
        p = replace(base, nx=w + 40, trench_w=w, trench_d=d, trench_taper_deg=taper, floor_t=10, mask_t=20,
                    n_vac=50, mask_type=mask, mask_eps_r=3.0, field_mode="floating", bias="rf",
                    electron_temp_eV=3.0, sigma_s=1e-15, n_per_batch=n, seed=int(rng.integers(1 << 30)))
        try:
            geometry.build_geometry(p)
        except ValueError:
            continue
        out.append(p)
        seps.append(sep)
    return out, seps


class ChargingBatch:
    """circuits: optional list with one circuit per case (None for a case without
    circuit_rf), as ChargingCase takes; RF cases trace with their in-flight clock in the
    same launch as the others.  claim_order: one of CLAIM_ORDERS for every case's queue
    (circuit_rf cases claim in index order under "learned")."""

    def __init__(self, params, device=0, green="f64", max_batches=None, circuits=None, claim_order="learned"):
        if not params:
            raise ValueError("a batch needs at least one case")
        circuits = [None] * len(params) if circuits is None else list(circuits)
        if len(circuits) != len(params):
            raise ValueError("one circuit (or None) per case")
        self.dev = torch.device("cuda", int(device))
        self.cases = [ChargingCase(p, device=device, precision="f32", green=green, max_batches=max_batches,
                                   circuit=c) for p, c in zip(params, circuits)]
        # the pack ends with the particles claimed last in every case: the learned order
        # (electrons first, then each case's ions longest predicted first, through the
        # batched ordering kernels) leaves the short ones for the end (64-case sweep: 13.7 ms
        # per batch in index order, 12.8 ms from the last particle down, 11.75 ms learned)
        if claim_order not in CLAIM_ORDERS:
            raise ValueError(f"claim_order must be one of {CLAIM_ORDERS}")
        for c in self.cases:
            c.set_claim_order(CLAIM_ORDERS.index(claim_order))
        L = _capi.lib()
        handles = (ctypes.c_void_p * len(self.cases))(*[c.ctx.handle.value for c in self.cases])
        h = ctypes.c_void_p()
        code = L.tb_pack_create(ctypes.byref(h), len(self.cases), handles)
        if code != _capi.TB_OK:
            _capi.raise_for(code, None)
        self.pack = h
        self.n_loaded = [0] * len(self.cases)
        self._graph = None
        self._args_for = None
        descs = (_capi.StepDesc * len(self.cases))(*[c._desc for c in self.cases])
        self._check(L.tb_pack_set_steps(self.pack, descs))
        self.per_case_update = False   # True: 3 launches per case (tb_step_charge, tb_step_potential)
        self.trace_events = None       # optional (start, end) CUDA events around the tracer launch

    def _check(self, code):
        if code != _capi.TB_OK:
            msg = _capi.lib().tb_pack_last_error(self.pack).decode(errors="replace")
            if code == _capi.TB_ERR_ARG:
                raise ValueError(msg)
            raise _capi.TBError(code, msg)

    def close(self):
        if getattr(self, "pack", None):
            _capi.lib().tb_pack_destroy(self.pack)
            self.pack = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, i, x, y, vx, vy, qm, spc, non_blocking=False, launch_times=None):
        self.cases[i].load(x, y, vx, vy, qm, spc, non_blocking=non_blocking, launch_times=launch_times)
        self.n_loaded[i] = len(x)

    def _set_args(self):
        key = tuple(self.n_loaded)
        if self._args_for == key:
            return
        arr = (_capi.TraceArgs * len(self.cases))()
        for i, (c, n) in enumerate(zip(self.cases, self.n_loaded)):
            # the case's own tracer arguments (fields, barrier, RF clock) for buffer set 0
            c._fill_args(n, 0)
            arr[i] = c._args
        self._check(_capi.lib().tb_pack_set_args(self.pack, arr))
        self._args_for = key

    def step(self):
        """One batch of every case on the current stream."""
        L = _capi.lib()
        self._set_args()
        s = ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        ev = self.trace_events
        if ev is not None:
            ev[0].record()
        self._check(L.tb_pack_trace(self.pack, 1, s))
        if ev is not None:
            ev[1].record()
        if self.per_case_update:
            for c in self.cases:
                c.ctx.check(L.tb_step_charge(c.ctx.handle, ctypes.byref(c._desc), s))
                c.ctx.check(L.tb_step_potential(c.ctx.handle, ctypes.byref(c._desc), s))
        else:
            self._check(L.tb_pack_step(self.pack, s))

    def capture(self):
        self._set_args()
        side = torch.cuda.Stream(self.dev)
        side.wait_stream(torch.cuda.current_stream(self.dev))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            with torch.cuda.graph(g, stream=side):
                self.step()
        torch.cuda.current_stream(self.dev).wait_stream(side)
        self._graph = g
        return g

    def replay(self):
        self._graph.replay()

    def check(self):
        s = ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        self._check(_capi.lib().tb_pack_check(self.pack, s))
        for c in self.cases:
            c.check()
