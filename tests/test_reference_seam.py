"""The reference's own batch loop driving this backend's tracer interface through its
tracer seam.

The reference selects its GPU tracer by importing ``trench_cuda.CudaTracer`` inside
make_particle_tracer (trench_charging_2d.py:705-724), and its tests patch that name
(tests/test_cuda.py:35-47).  Here the name is patched with B200Tracer's Python layer --
its argument checks, array handling, record and stop handling and return types -- with
only the device call replaced by the oracle, so that the reference's run() and
probe_vertical_ions() run on this host and must give exactly what they give with their
own CPU tracer (the oracle equals it bit for bit).  The kernels behind that layer are
checked against the reference's outputs in the GPU tests.

The reference is Python and present only where the fixtures are generated; on a machine
without it (the GPU box) these tests skip.
"""
import inspect
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def _reference():
    import __graft_entry__
    tree = __graft_entry__.reference_tree()
    if tree is None:
        pytest.skip("the reference source tree is not present on this machine")
    from make_golden import import_reference
    T, _ = import_reference(tree)
    import trench_cuda
    return T, trench_cuda


class OracleBackedTracer:
    """B200Tracer's interface layer with the device call replaced by the oracle."""

    def __new__(cls, vac, device=0):
        from oracle import oracle_trace
        from trench_b200.tracer import B200Tracer

        class Seam(B200Tracer):
            def __init__(self, vac, device=0):
                self.vac = np.asarray(vac, dtype=bool).copy()
                self.device = int(device)
                self.name = "oracle-backed interface"
                self.precision = "f64"
                self.calls = 0

            def _trace(self, x, y, vx, vy, qm, spc_h, Ex, Ey, p, barrier, record, stop, rf):
                self.calls += 1
                return oracle_trace.trace(x, y, vx, vy, qm, spc_h, Ex, Ey, self.vac, p, barrier, record=record,
                                          stop=stop, rf=rf)
        return Seam(vac, device)


def test_the_call_signature_is_the_reference_tracers():
    _, C = _reference()
    from trench_b200.tracer import B200Tracer
    ref, mine = inspect.signature(C.CudaTracer.__call__), inspect.signature(B200Tracer.__call__)
    assert [(q.name, q.default) for q in ref.parameters.values()] == \
           [(q.name, q.default) for q in mine.parameters.values()]
    ref_init = list(inspect.signature(C.CudaTracer.__init__).parameters.values())[:3]
    mine_init = list(inspect.signature(B200Tracer.__init__).parameters.values())[:3]
    assert [(q.name, q.default) for q in ref_init] == [(q.name, q.default) for q in mine_init]


def test_reference_run_through_the_seam_equals_its_cpu_run(monkeypatch):
    T, C = _reference()
    made = []

    def factory(vac, device=0):
        t = OracleBackedTracer(vac, device)
        made.append(t)
        return t
    monkeypatch.setattr(C, "CudaTracer", factory)
    base = dict(nx=30, trench_w=10, trench_d=24, floor_t=6, mask_t=8, n_vac=14, n_per_batch=600, n_batches=4,
                sigma_s=1e-14, trench_taper_deg=3.0, seed=4)
    cpu = T.run(replace(T.Params(), backend="cpu", **base), log=lambda s: None)
    seam = T.run(replace(T.Params(), backend="cuda", **base), log=lambda s: None)
    assert seam["backend_used"] == "cuda" and made and made[0].calls == base["n_batches"]
    np.testing.assert_array_equal(seam["rho_raw"], cpu["rho_raw"])
    np.testing.assert_array_equal(seam["mean_phi"], cpu["mean_phi"])
    for k in ("ratio_i_bottom", "ratio_e_bottom", "esc_e", "lost"):
        np.testing.assert_array_equal(seam["hist"][k], cpu["hist"][k])


def test_reference_probe_through_the_seam_records_like_its_cpu_probe(monkeypatch):
    T, C = _reference()
    monkeypatch.setattr(C, "CudaTracer", OracleBackedTracer)
    p = replace(T.Params(), nx=30, trench_w=10, trench_d=24, floor_t=6, mask_t=8, n_vac=14, sigma_s=0, bias="dc",
                probe_ions=60, probe_trajectories=6, max_steps=600)
    solid, mask, _, _ = T.build_geometry(p)
    res = dict(params=dict(vars(p)) if not hasattr(p, "__dataclass_fields__") else __import__("dataclasses").asdict(p),
               solid=solid, mask=mask, rho_raw=np.zeros(solid.shape), t_conv=1e-3, stopped=False)
    cpu = T.probe_vertical_ions(res, replace(p, backend="cpu"), log=lambda s: None)
    seam = T.probe_vertical_ions(res, replace(p, backend="cuda"), log=lambda s: None)
    assert seam["backend_used"] == "cuda"
    for label in ("charged", "uncharged"):
        a, b = seam[label], cpu[label]
        for k in ("hits", "status", "hit_cells", "endpoints", "final_velocity", "angle_deg"):
            np.testing.assert_array_equal(a[k], b[k])
        assert [len(v) for v in a["paths"]] == [len(v) for v in b["paths"]]
