"""Surface leakage on the device conserves charge and spreads it over a connected
surface (the reference's tests/test_taper.py:112-130, restated for this backend's
leakage operator and its in-place application by the batch step)."""
from dataclasses import replace

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_leakage_is_connected_and_conserves_charge_on_steps(cuda_device):
    import torch
    from scipy.sparse.csgraph import connected_components
    from trench_b200 import geometry
    from trench_b200.step import ChargingCase
    p = replace(load_golden("run_taper_leak.npz")["p"], sigma_s=1e-14, mask_type="dielectric", n_batches=2)
    case = ChargingCase(p, device=cuda_device, max_batches=4)
    G = case.leak_G
    assert connected_components(G, directed=False)[0] == 1
    np.testing.assert_allclose(G.sum(axis=0), 0, atol=1e-20)
    # one source cell at the bottom centre: the operator keeps the total and spreads it
    b0, b1 = geometry.opening_span(case.solid, p.floor_t)
    src = int(np.flatnonzero(case.S == ((b0 + b1) // 2) * case.ny + p.floor_t - 1)[0])
    q = np.zeros(case.m)
    q[src] = 1e-12
    after = case.leak_M.cpu().numpy() @ q
    assert after.sum() == pytest.approx(q.sum(), rel=1e-12)
    assert np.count_nonzero(np.abs(after) > 1e-18) > 2
    # the batch step applies it on the device: batches without particles keep the total
    case.rho_s.zero_()
    case.rho_s[src] = q[src] / p.dx ** 2
    total0 = float(case.rho_s.sum()) * p.dx ** 2
    for _ in range(2):
        case.step(0)
    torch.cuda.synchronize()
    case.check()
    rho = case.rho_s.cpu().numpy()
    assert rho.sum() * p.dx ** 2 == pytest.approx(total0, rel=1e-12)
    assert np.count_nonzero(np.abs(rho) > 1e-18 / p.dx ** 2) > 2
