"""The adjoint's FP64 PyTorch oracle: its surrogate recurrence at r = 1 equals the
reference batch loop (restated by BatchState, pinned to reference runs), and its
autograd gradient equals central finite differences of itself."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import oracle_adjoint as OA
from oracle import oracle_fields as OF
from oracle import oracle_trace as OT
from trench_b200 import geometry, inject


def surrogate_of(st, p, solid):
    """The oracle surrogate for a BatchState's case, slots in surface-cell order."""
    nx, ny = solid.shape
    sx, sy = np.nonzero(OF.surface_cells(solid))
    flat = sx * ny + sy
    sflag = np.zeros(len(flat), np.uint8)
    sflag[st.cond.ravel()[flat]] |= OA.SFLAG_COND
    sflag[(sy == p.floor_t - 1) & (sx >= st.b0) & (sx < st.b1)] |= OA.SFLAG_BOTTOM
    M = h = None
    if st.leak is not None:
        M = st.leak["M"]
        if np.any(st.fields["external"]):
            h = p.dt_batch * (st.leak["G"] @ st.fields["external"].ravel()[flat])
    g, c_slot, C = None, -1, 0.0
    if st.conductor:
        g = st.g_cond.ravel()[flat]
        c_slot = int(np.flatnonzero(flat == st.c_cell)[0])
        C = st.C_cond
    return OA.Surrogate(sflag, M, h, g, c_slot, st.conductor, st.driven, st.q_macro, p.dx, C,
                        p.electron_temp_eV), flat


def recorded_run(name, ne=4, na=3, seed=5):
    """Reference-loop run of a golden case; tables with the ion counts split into ne
    energy and na angle bins at random (each split sums to the ion count)."""
    g = load_golden(f"run_{name}.npz")
    p = g["p"]
    solid, mask, _, _ = geometry.build_geometry(p)
    st = OF.BatchState(p, solid, mask)
    sur, flat = surrogate_of(st, p, solid)
    rng = np.random.default_rng(p.seed)
    split = np.random.default_rng(seed)
    tables = []
    for _ in range(p.n_batches):
        parts = inject.inject(p, p.n_per_batch, solid.shape[1], rng)
        cnt_i, cnt_e, esc, lost = OT.trace(*parts, st.Ex, st.Ey, ~solid, p, st.barrier())
        ni, nel = cnt_i.ravel()[flat], cnt_e.ravel()[flat]
        TE = np.array([split.multinomial(k, np.ones(ne) / ne) for k in ni]).T
        TA = np.array([split.multinomial(k, np.ones(na) / na) for k in ni]).T
        tables.append(np.vstack([TE, TA, ni[None], nel[None]]))
        st.step(cnt_i, cnt_e, esc, lost)
    return p, st, sur, flat, np.array(tables)


@pytest.mark.parametrize("name", ["floating_leak", "fixed_leak", "dielectric_leak", "floating_noleak"])
def test_surrogate_at_unit_weights_is_the_reference_loop(name):
    p, st, sur, flat, tables = recorded_run(name)
    ne, na = 4, 3
    one = lambda k: torch.ones(k, dtype=torch.float64)
    rho, bottom = sur.run(tables, ne, na, one(ne), one(na), torch.zeros(len(flat), dtype=torch.float64))
    scale = np.abs(st.rho).max()
    np.testing.assert_allclose(rho.numpy(), st.rho.ravel()[flat], rtol=1e-12, atol=1e-12 * scale)
    norm = p.n_per_batch * (st.b1 - st.b0) / p.nx
    np.testing.assert_allclose(bottom.numpy() / norm, st.hist["ratio_i_bottom"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("with_feedback", [False, True])
def test_oracle_gradient_matches_its_finite_differences(with_feedback):
    p, st, sur, flat, tables = recorded_run("floating_leak")
    ne, na, m = 4, 3, len(flat)
    fb = None
    if with_feedback:
        # a made-up linear response along 3 orthonormal modes
        r = np.random.default_rng(3)
        V = torch.as_tensor(np.linalg.qr(r.normal(size=(m, 3)))[0])
        scale = 1.0 / np.abs(st.rho).max()
        fb = (V, torch.as_tensor(r.normal(size=(2, m, 3)) * scale), torch.as_tensor(r.normal(size=(2, m, 3)) * scale),
              torch.as_tensor([0, 0, 1, 1]))
    c = np.random.default_rng(1).normal(size=m)

    def J(rE, rA, rho0):
        rho, bottom = sur.run(tables, ne, na, rE, rA, rho0, feedback=fb)
        return (torch.as_tensor(c) * rho).sum() * 1e3 + bottom[-1] / 50.0

    rE = torch.ones(ne, dtype=torch.float64, requires_grad=True)
    rA = torch.ones(na, dtype=torch.float64, requires_grad=True)
    rho0 = torch.zeros(m, dtype=torch.float64, requires_grad=True)
    J(rE, rA, rho0).backward()
    one_e, one_a = torch.ones(ne, dtype=torch.float64), torch.ones(na, dtype=torch.float64)
    if not with_feedback:
        # without feedback the objective is a function of r: its differences pin the gradient
        h = 1e-6
        for k in range(ne):
            e = torch.zeros(ne, dtype=torch.float64)
            e[k] = h
            with torch.no_grad():
                fd = (J(1 + e, one_a, rho0) - J(1 - e, one_a, rho0)) / (2 * h)
            assert abs(fd.item() - rE.grad[k].item()) <= 1e-6 * abs(rE.grad).max().item()
        v = torch.as_tensor(np.random.default_rng(2).normal(size=m)) * np.abs(st.rho).max()
        with torch.no_grad():
            fd = (J(one_e, one_a, rho0 + 1e-6 * v) - J(one_e, one_a, rho0 - 1e-6 * v)) / 2e-6
        np.testing.assert_allclose(fd.item(), (rho0.grad * v).sum().item(), rtol=1e-6)
    else:
        # with feedback the gradient is that of the linearised chain, whose deposits move
        # with the state: ci_b(rho) = ci_b + Ri V^T (rho - rho_b), rho_b the base run's
        # states (constants here).  That is an ordinary function of (r, rho0), so its
        # central differences pin the gradient.
        with torch.no_grad():
            base, states = torch.zeros(m, dtype=torch.float64), []
            for b in range(len(tables)):
                states.append(base.clone())
                base, _ = sur.run(tables[b:b + 1], ne, na, one_e, one_a, base)

        def J_lin(rE_, rA_, rho0_):
            rho, bottom = rho0_, None
            for b in range(len(tables)):
                T = torch.as_tensor(tables[b], dtype=torch.float64).clone()
                d = fb[0].T @ (rho - states[b])
                T[ne + na] = T[ne + na] + fb[1][int(fb[3][b])] @ d
                T[ne + na + 1] = T[ne + na + 1] + fb[2][int(fb[3][b])] @ d
                ci = T[ne + na] + (rE_ - 1.0) @ T[:ne] + (rA_ - 1.0) @ T[ne:ne + na]
                T2 = torch.stack([ci, T[ne + na + 1]])[None]      # no bins: all ions, electrons
                rho, bottom = sur.run(T2.numpy(), 0, 0, torch.ones(0, dtype=torch.float64),
                                      torch.ones(0, dtype=torch.float64), rho)
            return (torch.as_tensor(c) * rho).sum() * 1e3 + bottom[-1] / 50.0

        h = 1e-6
        with torch.no_grad():
            for k in range(ne):
                e = torch.zeros(ne, dtype=torch.float64)
                e[k] = h
                fd = (J_lin(1 + e, one_a, rho0) - J_lin(1 - e, one_a, rho0)) / (2 * h)
                assert abs(fd.item() - rE.grad[k].item()) <= 1e-5 * abs(rE.grad).max().item()
            v = torch.as_tensor(np.random.default_rng(2).normal(size=m)) * np.abs(st.rho).max()
            fd = (J_lin(one_e, one_a, rho0 + 1e-6 * v) - J_lin(one_e, one_a, rho0 - 1e-6 * v)) / 2e-6
        np.testing.assert_allclose(fd.item(), (rho0.grad * v).sum().item(), rtol=1e-5)
