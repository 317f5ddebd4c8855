"""ORACLE -- test infrastructure only (the checker, never the product).

Drives the reference's own FP64 CUDA kernel ``trace_particles``
(trench_trace.cu:70-193), compiled unmodified for sm_100a into
``_ref/trench_trace.cubin`` by ``make -C oracle ref``, exactly the way the
reference's host wrapper does (trench_cuda.py:50-138): particles packed AoS
(n x 5 FP64) and fields copied to the device on every call, 128-thread blocks,
256-step chunks with a host synchronisation after each chunk, hits counted with
a host bincount.  This is the plain single-case FP64 GPU form the B200 backend is
measured against.  CuPy (the reference's launcher) is not installed, so device
memory comes from torch and the kernel is launched through the CUDA driver API.
"""
import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
CUBIN = HERE / "_ref" / "trench_trace.cubin"

_cu = None


def _driver():
    global _cu
    if _cu is None:
        cu = ctypes.CDLL("libcuda.so.1")
        cu.cuInit.argtypes = [ctypes.c_uint]
        cu.cuDeviceGet.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        cu.cuDevicePrimaryCtxRetain.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
        cu.cuCtxSetCurrent.argtypes = [ctypes.c_void_p]
        cu.cuModuleLoad.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p]
        cu.cuModuleGetFunction.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_char_p]
        cu.cuLaunchKernel.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                      ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint,
                                      ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]
        _cu = cu
    return _cu


def available():
    return CUBIN.exists()


class RefCudaTracer:
    """The reference CUDA tracer call (trench_cuda.py:41-138) without record, with the RF
    in-flight clock (trench_cuda.py:62-72)."""

    def __init__(self, vac, device=0):
        import torch
        if not CUBIN.exists():
            raise RuntimeError(f"{CUBIN} is not built (make -C oracle ref)")
        self.torch = torch
        self.dev = torch.device("cuda", device)
        torch.zeros(1, device=self.dev)          # runtime initialises the primary context
        cu = _driver()
        chk = lambda r, what: (_ for _ in ()).throw(RuntimeError(f"{what} failed ({r})")) if r else None
        chk(cu.cuInit(0), "cuInit")
        d = ctypes.c_int()
        chk(cu.cuDeviceGet(ctypes.byref(d), device), "cuDeviceGet")
        ctx = ctypes.c_void_p()
        chk(cu.cuDevicePrimaryCtxRetain(ctypes.byref(ctx), d), "cuDevicePrimaryCtxRetain")
        chk(cu.cuCtxSetCurrent(ctx), "cuCtxSetCurrent")
        mod = ctypes.c_void_p()
        chk(cu.cuModuleLoad(ctypes.byref(mod), str(CUBIN).encode()), "cuModuleLoad")
        fn = ctypes.c_void_p()
        chk(cu.cuModuleGetFunction(ctypes.byref(fn), mod, b"trace_particles"), "cuModuleGetFunction")
        self.fn = fn
        self.vac = np.asarray(vac, dtype=bool).copy()
        self.gpu_vac = torch.from_numpy(self.vac.astype(np.uint8)).to(self.dev)
        self.dummy = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.dummy_int = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.launches = 0

    def _launch(self, grid, args):
        holders, ptrs = [], []
        for kind, v in args:
            if kind == "p":
                h = ctypes.c_void_p(v)
            elif kind == "i":
                h = ctypes.c_int(v)
            else:
                h = ctypes.c_double(v)
            holders.append(h)
            ptrs.append(ctypes.cast(ctypes.pointer(h), ctypes.c_void_p))
        arr = (ctypes.c_void_p * len(ptrs))(*[p.value for p in ptrs])
        stream = self.torch.cuda.current_stream(self.dev).cuda_stream
        r = _driver().cuLaunchKernel(self.fn, grid, 1, 1, 128, 1, 1, 0, ctypes.c_void_p(stream), arr, None)
        if r:
            raise RuntimeError(f"cuLaunchKernel failed ({r})")
        self.launches += 1

    def __call__(self, x, y, vx, vy, qm, spc, Ex, Ey, vac, p, barrier=None, rf=None):
        torch = self.torch
        if vac.shape != self.vac.shape or not np.array_equal(vac, self.vac):
            raise ValueError("geometry changed")
        n = len(x)
        nx, ny = self.vac.shape
        dev = self.dev
        # trench_cuda.py:60-61, 73-80: per-call host-to-device copies
        particles = torch.from_numpy(np.column_stack((x, y, vx, vy, qm)).astype(np.float64)).to(dev)
        ex = torch.from_numpy(np.ascontiguousarray(Ex, dtype=np.float64)).to(dev)
        ey = torch.from_numpy(np.ascontiguousarray(Ey, dtype=np.float64)).to(dev)
        status = torch.full((n,), 3, dtype=torch.int8, device=dev)
        hits = torch.full((n,), -1, dtype=torch.int32, device=dev)
        if barrier is None:
            phi = wface = self.dummy
        else:
            phi = torch.from_numpy(np.ascontiguousarray(barrier[0], dtype=np.float64)).to(dev)
            wface = torch.from_numpy(np.ascontiguousarray(barrier[1], dtype=np.float64)).to(dev)
        tapered = int(bool(p.trench_taper_deg or (p.mask_t > 0 and p.mask_taper_deg)))
        d64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
        if rf is None:
            rf_ex = rf_ey = rf_phi = wave = clocks = self.dummy
            period, dt_max, n_phase, bound = 1.0, 1.0, 0, np.zeros(2)
        else:
            rf_ex, rf_ey, rf_phi, wave = (d64(rf[k]) for k in ("Ex", "Ey", "phi", "wave"))
            clocks = d64(np.column_stack((np.asarray(rf["initial_time"]) % rf["period"], np.zeros(n))))
            period, dt_max, n_phase = float(rf["period"]), float(rf["dt_max"]), len(rf["wave"])
            bound = np.abs(np.asarray(rf["wave"])).max(axis=0)
        host_status = np.full(n, 3, dtype=np.int8)
        dp = lambda t: t.data_ptr()
        for offset in range(0, p.max_steps, 256):               # trench_cuda.py:100-117
            if not n or not np.any(host_status == 3):
                break
            args = [("p", dp(particles)), ("p", dp(ex)), ("p", dp(ey)), ("p", dp(self.gpu_vac)),
                    ("p", dp(phi)), ("p", dp(wface)), ("p", dp(status)), ("p", dp(hits)),
                    ("p", dp(self.dummy)), ("p", dp(self.dummy_int)), ("p", dp(self.dummy)),
                    ("p", dp(self.dummy_int)),
                    ("p", dp(rf_ex)), ("p", dp(rf_ey)), ("p", dp(rf_phi)), ("p", dp(wave)), ("p", dp(clocks)),
                    ("i", n), ("i", nx), ("i", ny), ("i", min(256, p.max_steps - offset)), ("i", int(offset == 0)),
                    ("i", int(barrier is not None)), ("i", 0), ("i", tapered), ("i", p.max_steps + 1),
                    ("d", float(p.dx)), ("d", float(p.cfl)), ("i", n_phase), ("d", period), ("d", dt_max),
                    ("d", float(bound[0])), ("d", float(bound[1]))]
            self._launch((n + 127) // 128, args)
            host_status = status.cpu().numpy()                   # synchronises, once per chunk
        host_hits = hits.cpu().numpy()
        spc = np.asarray(spc)
        counts = [np.bincount(host_hits[(host_status == 1) & (spc == k)], minlength=nx * ny).reshape(nx, ny)
                  for k in (0, 1)]
        escaped = np.bincount(spc[host_status == 2], minlength=2).astype(np.int64)
        lost = int(np.count_nonzero(host_status == 3))
        return counts[0], counts[1], escaped, lost
