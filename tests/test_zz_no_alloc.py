"""The no-allocation FP32 tracer entry point against the context-based one.

tb_trace_f32_noalloc serves callers that cannot call cudaMalloc (a host
application whose pool owns all device memory, or code that must not let an
allocation synchronise the device): its scratch is a static device array.  This
file is collected last so that, in a run stopping at the first failure, every
other test has already run; it passes alone in a fresh process too.

Cases: the charged AR-8 geometry (its packed field fits in shared memory), a
256 x 256 grid at the cell limit (field read from global memory) and a 1 x 65536
strip, whose halo-padded field is the largest the static array holds.
"""
import ctypes
from dataclasses import replace

import numpy as np
import pytest

from conftest import load_golden
from trench_b200 import inject

pytestmark = pytest.mark.gpu


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def noalloc_trace(device, parts, vac, Ex, Ey, p, barrier, vscale):
    """Traces `parts` twice in a row through tb_trace_f32_noalloc; returns each call's
    (counts, escaped, lost, particle-steps)."""
    import torch
    from trench_b200 import _capi
    from trench_b200.params import is_tapered
    nx, ny = vac.shape
    n = len(parts[0])
    dev = torch.device("cuda", device)
    f64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    VAC = torch.from_numpy(np.ascontiguousarray(vac, dtype=np.uint8)).to(dev)
    EX, EY = f64(Ex), f64(Ey)
    PHI, WF = (f64(barrier[0]), f64(barrier[1])) if barrier is not None else (None, None)
    L = _capi.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    out = []
    for _ in range(2):  # two calls in a row share the static scratch
        X = [f64(v) for v in parts[:5]]
        SPC = torch.from_numpy(np.ascontiguousarray(parts[5], dtype=np.int8)).to(dev)
        counts = torch.zeros((2, nx, ny), dtype=torch.int32, device=dev)
        totals = torch.full((8,), -1, dtype=torch.int64, device=dev)
        totals[:6] = 0
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
        code = L.tb_trace_f32_noalloc(nx, ny, float(p.dx), _ptr(VAC), ctypes.byref(a), vscale, stream)
        assert code == 0, L.tb_last_error(None)
        torch.cuda.synchronize()
        tot = totals.cpu().numpy()
        assert tot[6] == 0, "device check flag raised"
        out.append((counts.to(torch.int64).cpu().numpy(), tot[:2].copy(),
                    int(np.count_nonzero(status.cpu().numpy() == 3)), int(tot[3])))
    return out


def check_against_context(device, parts, vac, Ex, Ey, p, barrier):
    from trench_b200.tracer import B200Tracer
    tracer = B200Tracer(vac, device, precision="f32")
    want = tracer(*parts, Ex, Ey, vac, p, barrier)
    want_steps = tracer.last["particle_steps"]
    for cnt, esc, lost, steps in noalloc_trace(device, parts, vac, Ex, Ey, p, barrier, tracer.vscale):
        np.testing.assert_array_equal(cnt[0], want[0])
        np.testing.assert_array_equal(cnt[1], want[1])
        np.testing.assert_array_equal(esc, want[2])
        assert lost == want[3]
        assert steps == want_steps
    return want


def test_noalloc_trace_matches_context_trace(cuda_device):
    g = load_golden("trace_cfg2.npz")  # charged AR-8 geometry, tapered walls, barrier model
    p = g["p"]
    solid = g["solid"]
    parts = inject.inject(p, 1 << 14, solid.shape[1], np.random.default_rng(77))
    check_against_context(cuda_device, parts, ~solid, g["Ex"], g["Ey"], p, (g["phi"], g["wface"]))


def synthetic_case(nx, ny, floor, n, seed, pillar=False):
    """A grid of nx x ny cells with `floor` solid rows (and optionally a solid pillar
    in the middle columns), a smooth field pulling ions down, a smooth wall potential,
    and n ions + n electrons started uniformly in the vacuum."""
    from trench_b200.params import Params
    rng = np.random.default_rng(seed)
    solid = np.zeros((nx, ny), dtype=bool)
    solid[:, :floor] = True
    if pillar:
        solid[nx // 2 - nx // 8:nx // 2 + nx // 8, floor:floor + ny // 3] = True
    ix, iy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    phi = 5.0 * np.sin(2 * np.pi * ix / max(nx, 2)) * np.cos(np.pi * iy / ny) + 20.0 * iy / ny
    Ex = 1e6 * np.cos(2 * np.pi * ix / max(nx, 2) + 0.3) * np.exp(-iy / ny)
    Ey = -2e7 * (1.0 + 0.2 * np.sin(np.pi * iy / ny))
    Ex[solid] = Ey[solid] = 0.0
    p = replace(Params(), dx=5e-9, nx=nx, n_per_batch=n, max_steps=1500, cfl=0.35,
                trench_taper_deg=2.0, mask_taper_deg=0.0)
    x, y, vx, vy, qm, spc = inject.inject(p, n, ny, rng)
    y = rng.uniform(floor + 1, ny, size=2 * n) * p.dx
    x = rng.uniform(0.0, nx, size=2 * n) * p.dx
    return (x, y, vx, vy, qm, spc), ~solid, Ex, Ey, p, (phi, np.full((nx, ny), 0.75))


def test_noalloc_at_the_cell_limit_square_grid(cuda_device):
    """256 x 256 = TB_NOALLOC_MAX_CELLS: the packed field (532 KB) is read from global memory."""
    parts, vac, Ex, Ey, p, barrier = synthetic_case(256, 256, 40, 1 << 13, 3, pillar=True)
    want = check_against_context(cuda_device, parts, vac, Ex, Ey, p, barrier)
    assert want[0].sum() + want[1].sum() > 0  # walls were hit


def test_noalloc_at_the_field_bound_strip(cuda_device):
    """1 x 65536: the halo-padded field (3 x 65538 cells) reaches the static array's bound."""
    parts, vac, Ex, Ey, p, barrier = synthetic_case(1, 65536, 100, 1 << 12, 4)
    check_against_context(cuda_device, parts, vac, Ex, Ey, p, barrier)


def test_noalloc_rejects_oversized_grid(cuda_device):
    from trench_b200 import _capi
    L = _capi.lib()
    a = _capi.TraceArgs()
    a.n = 0
    a.cfl, a.max_steps, a.step_budget = 0.35, 10, 10
    code = L.tb_trace_f32_noalloc(300, 300, 1e-9, ctypes.c_void_p(1), ctypes.byref(a), 1e5, None)
    assert code == _capi.TB_ERR_ARG
    assert b"exceeds" in L.tb_last_error(None)


def test_noalloc_empty_batch_clears_the_flag_slot(cuda_device):
    """n = 0 traces nothing and still writes 0 to totals[6]."""
    import torch
    from trench_b200 import _capi
    L = _capi.lib()
    dev = torch.device("cuda", cuda_device)
    totals = torch.full((8,), 7, dtype=torch.int64, device=dev)
    vac = torch.ones(16, dtype=torch.uint8, device=dev)
    a = _capi.TraceArgs()
    a.n = 0
    a.cfl, a.max_steps, a.step_budget = 0.35, 10, 10
    a.d_totals = _ptr(totals)
    code = L.tb_trace_f32_noalloc(4, 4, 1e-9, _ptr(vac), ctypes.byref(a), 1e5,
                                  ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    assert code == 0, L.tb_last_error(None)
    torch.cuda.synchronize()
    assert totals.cpu().numpy().tolist() == [7, 7, 7, 7, 7, 7, 0, 7]
