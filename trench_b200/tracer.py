"""B200Tracer: the reference tracer interface on the sm_100a kernels.

``B200Tracer(vac, device)`` is called exactly like the reference
``CudaTracer`` (trench_cuda.py:21-138) and ``trace_cpu``
(trench_charging_2d.py:542):

    cnt_i, cnt_e, escaped, lost = tracer(x, y, vx, vy, qm, spc, Ex, Ey, vac, p,
                                         barrier=None, record=None, stop=None, rf=None)

Inputs are host NumPy arrays (any memory order) or CUDA torch tensors; the
outputs are new NumPy arrays.  ``precision="f32"`` runs the FP32 shared-memory
kernel; ``"f64"`` runs the reference-exact FP64 kernel.  Both carry the RF
in-flight clock; trajectory recording always uses the FP64 kernel.  There is no
CPU path.
"""
import ctypes
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import _capi
from .params import is_tapered

CHUNK_STEPS = 256      # step budget per launch when a stop event must be polled
DEFAULT_VSCALE = 1e5   # m/s, velocity unit of the FP32 state


class _HostStager:
    """Host-to-device copies of large pageable host arrays through two pinned staging
    buffers: worker threads copy chunk k+1 into one buffer (NumPy copies release the
    interpreter lock, so the host copy runs at several threads' bandwidth) while the copy
    engine moves chunk k from the other, on a copy stream that the caller's stream then
    waits for.  A plain pageable copy runs at one host thread's memcpy rate."""

    CHUNK = 8 << 20

    def __init__(self, device):
        self.dev = device
        self.pinned = [torch.empty(self.CHUNK, dtype=torch.uint8).pin_memory() for _ in range(2)]
        self.host = [t.numpy() for t in self.pinned]
        self.stream = torch.cuda.Stream(device)
        self.events = [None, None]
        self.k = 0
        self.threads = max(1, min(8, os.cpu_count() or 1))
        self.pool = ThreadPoolExecutor(self.threads) if self.threads > 1 else None

    def _fill(self, dst, src):
        n = src.size
        if self.pool is None or n < (1 << 20):
            np.copyto(dst, src)
            return
        step = -(-n // self.threads)
        list(self.pool.map(lambda i: np.copyto(dst[i * step:(i + 1) * step], src[i * step:(i + 1) * step]),
                           range(self.threads)))

    def copy(self, dst, src):
        """dst: contiguous 1-D device tensor; src: contiguous host array of dst's bytes."""
        sb = src.reshape(-1).view(np.uint8)
        db = dst.view(torch.uint8)
        for off in range(0, sb.size, self.CHUNK):
            j = self.k % 2
            self.k += 1
            ln = min(self.CHUNK, sb.size - off)
            if self.events[j] is not None:
                self.events[j].synchronize()        # the buffer's previous chunk has been copied
            self._fill(self.host[j][:ln], sb[off:off + ln])
            with torch.cuda.stream(self.stream):
                db[off:off + ln].copy_(self.pinned[j][:ln], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.stream)
            self.events[j] = ev

    def join(self):
        """The current stream waits for every copy issued so far."""
        torch.cuda.current_stream(self.dev).wait_stream(self.stream)


def _validate_rf(rf, n, shape):
    """trench_rf.py:21-32"""
    if (not np.isfinite(rf["period"]) or rf["period"] <= 0
            or not np.isfinite(rf["dt_max"]) or rf["dt_max"] <= 0):
        raise ValueError("RF period and dt_max must be positive and finite")
    for key in ("phi", "Ex", "Ey"):
        if np.shape(rf[key]) != (2, *shape) or not np.isfinite(rf[key]).all():
            raise ValueError("RF basis field has a wrong shape or non-finite values")
    wave = np.asarray(rf["wave"])
    if wave.ndim != 2 or wave.shape[1] != 2 or len(wave) < 2 or not np.isfinite(wave).all():
        raise ValueError("RF voltage waveform is invalid")
    if np.shape(rf["initial_time"]) != (n,) or not np.isfinite(rf["initial_time"]).all():
        raise ValueError("particle launch times have a wrong shape or non-finite values")


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class Context:
    """Owns one tb_ctx (one grid and vacuum mask on one device)."""

    def __init__(self, vac, device=0, dx=1.0):
        L = _capi.lib()
        vac = np.ascontiguousarray(np.asarray(vac, dtype=bool), dtype=np.uint8)
        self.nx, self.ny = vac.shape
        h = ctypes.c_void_p()
        code = L.tb_create(ctypes.byref(h), int(device), self.nx, self.ny, float(dx),
                           vac.ctypes.data_as(ctypes.c_void_p))
        if code == _capi.TB_ERR_DEVICE:
            msg = L.tb_last_error(None).decode()
            raise RuntimeError(f"{msg} (CUDA デバイス {device} は利用できません)")
        _capi.raise_for(code, None)
        self.handle = h
        self.device = int(device)
        buf = ctypes.create_string_buffer(128)
        sms = ctypes.c_int()
        L.tb_device_info(h, buf, 128, ctypes.byref(sms))
        self.name = buf.value.decode()
        self.num_sms = sms.value

    def check(self, code):
        _capi.raise_for(code, self.handle)

    def close(self):
        if getattr(self, "handle", None):
            _capi.lib().tb_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class B200Tracer:
    """Drop-in for ``CudaTracer`` (trench_cuda.py:21) running on the B200 kernels."""

    def __init__(self, vac, device=0, precision="f32", vscale=DEFAULT_VSCALE):
        if precision not in _capi.PRECISION:
            raise ValueError(f"precision must be one of {tuple(_capi.PRECISION)}")
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device is visible (the B200 backend has no CPU path)")
        self.vac = np.asarray(vac, dtype=bool).copy()
        self.ctx = Context(self.vac, device)
        self.device = self.ctx.device
        self.name = self.ctx.name
        self.precision = precision
        self.vscale = float(vscale)
        self.tdev = torch.device("cuda", self.device)
        self._stager = None       # pinned staging of large host arrays (created on first use)
        self._last_dev = None     # device outputs of the last call, read back on first use of .last
        self._last_host = {}
        self._ctx_dx = None
        self._bufs = {}           # device buffers kept between calls (particles, fields, outputs)
        self._field_host = None   # host copies of the last call's fields: unchanged fields are not re-sent
        self._field_dev = None
        self._packed = None       # vscale the context's FP32 field was last packed with

    @property
    def last(self):
        """Per-particle outputs of the last call (status, absorbing cell, steps) and its
        particle-step total; copied to the host when first asked for."""
        if self._last_dev is not None:
            d = self._last_dev
            self._last_host = dict(particle_steps=d["particle_steps"], precision=d["precision"],
                                   status=d["status"].cpu().numpy(), hit=d["hit"].cpu().numpy(),
                                   steps=d["steps"].cpu().numpy())
            self._last_dev = None
        return self._last_host

    # -- helpers ---------------------------------------------------------------
    def _dev(self, a, dtype):
        if isinstance(a, torch.Tensor):
            return a.to(device=self.tdev, dtype=dtype).contiguous()
        return torch.from_numpy(np.ascontiguousarray(a, dtype=_np_dtype(dtype))).to(self.tdev, non_blocking=False)

    def _buf(self, name, dtype, n):
        """The n-element view of the tracer's own device buffer `name`, grown to at
        least n elements when needed and kept between calls."""
        buf = self._bufs.get(name)
        if buf is None or buf.numel() < n:
            buf = torch.empty(max(n, 1), dtype=dtype, device=self.tdev)
            self._bufs[name] = buf
        return buf[:n]

    def _stage(self, name, src, dtype, n):
        """Copies `src` (host array or tensor, any memory order) into device buffer
        `name` (see _buf) and returns the view.  No allocation once the buffer is large
        enough."""
        view = self._buf(name, dtype, n)
        if isinstance(src, torch.Tensor):
            view.copy_(src.reshape(-1))
            return view
        host = np.ascontiguousarray(src, dtype=_np_dtype(dtype)).reshape(-1)
        if host.nbytes >= (1 << 20):
            if self._stager is None:
                self._stager = _HostStager(self.tdev)
            self._stager.copy(view, host)
            self._stager.join()
        else:
            view.copy_(torch.from_numpy(host))
        return view

    def _fields(self, Ex, Ey, barrier):
        """Device copies of the fields (and wall potential), uploaded only when they
        differ from the previous call's; returns (EX, EY, PHI, WF, changed)."""
        host = (Ex, Ey) + (tuple(barrier) if barrier is not None else ())
        host = tuple(a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, dtype=np.float64)
                     for a in host)
        last = self._field_host
        if last is not None and len(last) == len(host) and all(np.array_equal(a, b) for a, b in zip(host, last)):
            return (*self._field_dev, False)
        names = ("ex", "ey", "phi", "wface")
        dev = [self._stage(k, a, torch.float64, a.size) for k, a in zip(names, host)]
        dev += [None] * (4 - len(dev))
        self._field_host = tuple(a.copy() for a in host)
        self._field_dev = tuple(dev)
        return (*self._field_dev, True)

    def _context_for(self, dx):
        # The context stores dx; a tracer serves one geometry, dx comes from p.
        if self._ctx_dx != dx:
            self.ctx.close()
            self.ctx = Context(self.vac, self.device, dx)
            # FP32 launches claim in the learned order (electrons first, then ions longest
            # predicted first from the previous call): a call's time is set by the
            # particles still in flight when its queue runs dry
            self.ctx.check(_capi.lib().tb_set_claim_order(self.ctx.handle, 2))
            self._ctx_dx = dx
            self._packed = None
        return self.ctx

    # -- the reference call ------------------------------------------------------
    def __call__(self, x, y, vx, vy, qm, spc, Ex, Ey, vac, p, barrier=None, record=None, stop=None, rf=None):
        vac = np.asarray(vac)
        if vac.shape != self.vac.shape or not np.array_equal(vac.astype(bool), self.vac):
            raise ValueError("the tracer was built for another geometry; create a new tracer")
        if not (0 < p.cfl <= 1) or p.max_steps < 1:
            raise ValueError("CUDA tracing needs 0 < cfl <= 1 and max_steps >= 1")
        n = len(x)
        nx, ny = self.vac.shape
        if any(np.shape(v) != (n,) for v in (x, y, vx, vy, qm, spc)):
            raise ValueError("particle arrays differ in length")
        if any(np.shape(v) != (nx, ny) for v in (Ex, Ey)):
            raise ValueError("field shape does not match the grid")
        spc_h = spc.cpu().numpy() if isinstance(spc, torch.Tensor) else np.asarray(spc)
        if n and (spc_h.min() < 0 or spc_h.max() > 1 if spc_h.dtype.kind in "iub"
                  else np.any((spc_h != 0) & (spc_h != 1))):
            raise ValueError("species must be 0 (ion) or 1 (electron)")
        if barrier is not None and any(np.shape(v) != (nx, ny) for v in barrier):
            raise ValueError("wall potential shape does not match the grid")
        if record is not None and p.probe_trajectories < 1:
            raise ValueError("probe_trajectories must be at least 1")
        if rf is not None:
            _validate_rf(rf, n, self.vac.shape)
        return self._trace(x, y, vx, vy, qm, spc_h, Ex, Ey, p, barrier, record, stop, rf)

    def _trace(self, x, y, vx, vy, qm, spc_h, Ex, Ey, p, barrier, record, stop, rf):
        with torch.cuda.device(self.device):
            return self._trace_on_device(x, y, vx, vy, qm, spc_h, Ex, Ey, p, barrier, record, stop, rf)

    def _trace_on_device(self, x, y, vx, vy, qm, spc_h, Ex, Ey, p, barrier, record, stop, rf):
        L = _capi.lib()
        ctx = self._context_for(float(p.dx))
        n = len(x)
        nx, ny = self.vac.shape
        f64, dev = torch.float64, self.tdev
        precision = "f64" if record is not None else self.precision
        stream = torch.cuda.current_stream(dev)
        sp = ctypes.c_void_p(stream.cuda_stream)

        # particles go into the tracer's own buffers (the tracer writes particle state back
        # for record and at the step cap, so a caller's arrays are never traced in place)
        X = [self._stage(k, v, f64, n) for k, v in zip(("x", "y", "vx", "vy"), (x, y, vx, vy))]
        QM = self._stage("qm", qm, f64, n)
        SPC = self._stage("spc", spc_h, torch.int8, n)
        EX, EY, PHI, WF, fields_changed = self._fields(Ex, Ey, barrier)
        counts = self._bufs.get("counts")
        if counts is None:
            counts = self._bufs["counts"] = torch.empty((2, nx, ny), dtype=torch.int32, device=dev)
            self._bufs["totals"] = torch.empty(8, dtype=torch.int64, device=dev)
        totals = self._bufs["totals"]
        counts.zero_()
        totals.zero_()
        status = self._buf("status", torch.int8, n).fill_(3)
        hit = self._buf("hit", torch.int32, n).fill_(-1)
        steps = self._buf("steps", torch.int32, n).zero_()

        a = _capi.TraceArgs()
        a.n = n
        a.d_x, a.d_y, a.d_vx, a.d_vy = (_ptr(t) for t in X)
        a.d_qm, a.d_spc = _ptr(QM), _ptr(SPC)
        a.d_ex, a.d_ey = _ptr(EX), _ptr(EY)
        a.d_phi, a.d_wface = _ptr(PHI), _ptr(WF)
        a.max_steps = int(p.max_steps)
        a.cfl = float(p.cfl)
        a.tapered = int(is_tapered(p))
        a.d_counts, a.d_totals = _ptr(counts), _ptr(totals)
        a.d_status, a.d_hit, a.d_steps = _ptr(status), _ptr(hit), _ptr(steps)
        a.write_state = int(record is not None)

        keep = [X, QM, SPC, EX, EY, PHI, WF, counts, totals, status, hit, steps]
        period = None
        if rf is not None:
            RFX, RFY, RFP = (self._dev(rf[k], f64) for k in ("Ex", "Ey", "phi"))
            WAVE = self._dev(rf["wave"], f64)
            period = float(rf["period"])
            t0 = np.asarray(rf["initial_time"], dtype=np.float64) % period
            CLOCK = torch.from_numpy(np.column_stack((t0, np.zeros(n)))).to(dev)
            bound = np.abs(np.asarray(rf["wave"])).max(axis=0)
            a.d_rf_ex, a.d_rf_ey, a.d_rf_phi, a.d_wave = _ptr(RFX), _ptr(RFY), _ptr(RFP), _ptr(WAVE)
            a.n_phase = len(rf["wave"])
            a.period, a.dt_max = period, float(rf["dt_max"])
            a.bound_vs, a.bound_vm = float(bound[0]), float(bound[1])
            a.d_clock = _ptr(CLOCK)
            keep += [RFX, RFY, RFP, WAVE, CLOCK]
        selected = None
        if record is not None:
            selected = np.unique(np.linspace(0, n - 1, min(p.probe_trajectories, n), dtype=int))
            slots = np.full(n, -1, dtype=np.int32)
            slots[selected] = np.arange(len(selected), dtype=np.int32)
            stride = p.max_steps + 1
            SLOTS = torch.from_numpy(slots).to(dev)
            ENDP = torch.stack([X[0], X[1]], dim=1).contiguous()
            PATHS = torch.zeros((max(len(selected), 1), stride, 2), dtype=f64, device=dev)
            PLEN = torch.ones(max(len(selected), 1), dtype=torch.int32, device=dev)
            if len(selected):
                sel = torch.from_numpy(selected).to(dev)
                PATHS[:len(selected), 0] = ENDP[sel]
            a.record = 1
            a.d_endpoints, a.d_slots, a.d_paths, a.d_path_len = _ptr(ENDP), _ptr(SLOTS), _ptr(PATHS), _ptr(PLEN)
            a.path_stride = stride
            keep += [SLOTS, ENDP, PATHS, PLEN]

        if precision == "f32" and n:
            if fields_changed or self._packed != self.vscale:
                ctx.check(L.tb_set_fields(ctx.handle, _ptr(EX), _ptr(EY), _ptr(PHI), _ptr(WF), self.vscale, sp))
                self._packed = self.vscale
            if rf is not None:
                ctx.check(L.tb_set_rf_fields(ctx.handle, _ptr(RFX), _ptr(RFY), _ptr(RFP), _ptr(WF), _ptr(WAVE),
                                             len(rf["wave"]), sp))
        cancelled = False
        if stop is None:
            a.step_budget = int(p.max_steps)
            if n:
                ctx.check(L.tb_trace(ctx.handle, ctypes.byref(a), _capi.PRECISION[precision], sp))
        else:
            a.step_budget = min(CHUNK_STEPS, int(p.max_steps))
            for _ in range(0, int(p.max_steps), CHUNK_STEPS):
                if not n or not bool((status == 3).any()):
                    break
                if stop.is_set():
                    cancelled = True
                    break
                ctx.check(L.tb_trace(ctx.handle, ctypes.byref(a), _capi.PRECISION[precision], sp))
        ctx.check(L.tb_check(ctx.handle, sp))

        cnt = counts.cpu().numpy().astype(np.int64)
        tot = totals.cpu().numpy()
        escaped = np.array([tot[0], tot[1]], dtype=np.int64)
        # one launch over the whole step budget tallies the particles left live at the step
        # cap (totals[2]); chunked launches (a stop request) count the live status instead
        lost = int(tot[2]) if stop is None else int((status == 3).sum().item())
        self._last_dev = dict(particle_steps=int(tot[3]), status=status, hit=hit, steps=steps, precision=precision)
        if record is not None:
            host_status = self.last["status"]
            host_hit = self.last["hit"]
            cells = np.full((n, 2), -1, dtype=int)
            ab = host_status == 1
            cells[ab] = np.column_stack((host_hit[ab] // ny, host_hit[ab] % ny))
            plen = PLEN.cpu().numpy()
            paths = PATHS.cpu().numpy()
            record.update(selected=selected, status=host_status, hit_cells=cells,
                          initial_x=np.asarray(x).copy() if not isinstance(x, torch.Tensor) else x.cpu().numpy(),
                          endpoints=ENDP.cpu().numpy(),
                          final_velocity=np.column_stack((X[2].cpu().numpy(), X[3].cpu().numpy())),
                          paths=[paths[k, :plen[k]].copy() for k in range(len(selected))],
                          cancelled=cancelled or (stop is not None and stop.is_set()))
            if rf is not None:
                timing = CLOCK.cpu().numpy()
                record.update(launch_phase=np.asarray(rf["initial_time"]) % period / period * 360,
                              final_phase=timing[:, 0] / period * 360, flight_time=timing[:, 1])
        del keep
        return cnt[0], cnt[1], escaped, lost


def _np_dtype(tdtype):
    return {torch.float64: np.float64, torch.float32: np.float32, torch.int8: np.int8,
            torch.int32: np.int32, torch.int64: np.int64, torch.uint8: np.uint8}[tdtype]
