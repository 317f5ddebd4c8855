"""The no-allocation FP32 tracer entry point against the context-based one.

tb_trace_f32_noalloc serves callers that cannot call cudaMalloc (a host
application whose pool owns all device memory, or code that must not let an
allocation synchronise the device): its scratch is a static device array.  This
file is collected last so that, in a run stopping at the first failure, every
other test has already run; it passes alone in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_golden
from trench_b200 import inject

pytestmark = pytest.mark.gpu


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def test_noalloc_trace_matches_context_trace(cuda_device):
    import torch
    from trench_b200 import _capi
    from trench_b200.params import is_tapered
    from trench_b200.tracer import B200Tracer

    g = load_golden("trace_cfg2.npz")  # charged AR-8 geometry, tapered walls, barrier model
    p = g["p"]
    solid = g["solid"]
    nx, ny = solid.shape
    n_species = 1 << 14
    parts = inject.inject(p, n_species, ny, np.random.default_rng(77))
    n = 2 * n_species

    # existing entry point (context, tb_set_fields + tb_trace)
    tracer = B200Tracer(~solid, cuda_device, precision="f32")
    want = tracer(*parts, g["Ex"], g["Ey"], ~solid, p, (g["phi"], g["wface"]))
    want_steps = tracer.last["particle_steps"]

    dev = torch.device("cuda", cuda_device)
    f64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    vac = torch.from_numpy(np.ascontiguousarray(~solid, dtype=np.uint8)).to(dev)
    EX, EY, PHI, WF = f64(g["Ex"]), f64(g["Ey"]), f64(g["phi"]), f64(g["wface"])
    L = _capi.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    for call in range(2):  # two calls in a row share the static scratch
        X = [f64(v) for v in parts[:5]]
        SPC = torch.from_numpy(parts[5]).to(dev)
        counts = torch.zeros((2, nx, ny), dtype=torch.int32, device=dev)
        totals = torch.zeros(8, dtype=torch.int64, device=dev)
        status = torch.full((n,), 3, dtype=torch.int8, device=dev)
        steps = torch.zeros(n, dtype=torch.int32, device=dev)
        a = _capi.TraceArgs()
        a.n = n
        a.d_x, a.d_y, a.d_vx, a.d_vy, a.d_qm = (_ptr(t) for t in X)
        a.d_spc = _ptr(SPC)
        a.d_ex, a.d_ey, a.d_phi, a.d_wface = _ptr(EX), _ptr(EY), _ptr(PHI), _ptr(WF)
        a.max_steps = a.step_budget = int(p.max_steps)
        a.cfl = float(p.cfl)
        a.tapered = int(is_tapered(p))
        a.d_counts, a.d_totals, a.d_status, a.d_steps = _ptr(counts), _ptr(totals), _ptr(status), _ptr(steps)
        code = L.tb_trace_f32_noalloc(nx, ny, float(p.dx), _ptr(vac), ctypes.byref(a), tracer.vscale, stream)
        assert code == 0, L.tb_last_error(None)
        torch.cuda.synchronize()
        tot = totals.cpu().numpy()
        assert tot[6] == 0, "device check flag raised"
        cnt = counts.to(torch.int64).cpu().numpy()
        np.testing.assert_array_equal(cnt[0], want[0])
        np.testing.assert_array_equal(cnt[1], want[1])
        np.testing.assert_array_equal(tot[:2], want[2])
        assert int(np.count_nonzero(status.cpu().numpy() == 3)) == want[3]
        assert tot[3] == want_steps


def test_noalloc_rejects_oversized_grid(cuda_device):
    from trench_b200 import _capi
    L = _capi.lib()
    a = _capi.TraceArgs()
    a.n = 0
    a.cfl, a.max_steps, a.step_budget = 0.35, 10, 10
    code = L.tb_trace_f32_noalloc(300, 300, 1e-9, ctypes.c_void_p(1), ctypes.byref(a), 1e5, None)
    assert code == _capi.TB_ERR_ARG
    assert b"exceeds" in L.tb_last_error(None)
