"""Adjoint of the charging loop on the GPU: histories, surrogate replay, reverse
sweep and adjoint Poisson solve against the FP64 PyTorch oracle, finite
differences and the traced run itself."""
from dataclasses import replace

import numpy as np
import pytest

from oracle import oracle_adjoint as OA

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods(cuda_device):
    import torch
    from trench_b200 import adjoint, inject
    from trench_b200.step import ChargingCase
    return torch, adjoint, inject, ChargingCase


def record(mods, n=1 << 15, batches=12, k=5, seed=7, modes=0, **over):
    torch, adjoint, _, ChargingCase = mods
    p, eE, wE, eA, wA = adjoint.adjoint_workload(n_per_batch=n, n_batches=batches)
    p = replace(p, **over)
    case = ChargingCase(p, precision="f32", max_batches=batches)
    rec = adjoint.AdjointRecorder(case, eE, wE, eA, wA, seed=seed, checkpoint_every=k, feedback_modes=modes,
                                  feedback_every=k)
    return case, rec, rec.run(batches)


@pytest.fixture(scope="module")
def recorded(mods):
    return record(mods)


@pytest.fixture(scope="module")
def recorded_fb(mods):
    return record(mods, modes=6)


def oracle_of(case):
    d = case._desc
    return OA.Surrogate(case.t_sflag.cpu().numpy(), None if case.leak_M is None else case.leak_M.cpu().numpy(),
                        None if case.leak_h is None else case.leak_h.cpu().numpy(),
                        None if case.g_s is None else case.g_s.cpu().numpy(), case.c_slot, case.floating,
                        case.driven, d.q_macro, d.dx, d.C_cond, d.Te)


def probe_row(case):
    ix, iy = case.probes["bottom center"]
    return int(np.searchsorted(case.rows, ix * case.ny + iy)), ix * case.ny + iy


def test_injected_bins_are_the_tables_bins(mods):
    """The bin written for each ion is the bin its Philox draw falls in."""
    torch, adjoint, inject, ChargingCase = mods
    p, eE, wE, eA, wA = adjoint.adjoint_workload(n_per_batch=4096, n_batches=1)
    case = ChargingCase(p, precision="f32", max_batches=1)
    inj = inject.DeviceInjector(case, seed=11, energy_table=inject.histogram_table(eE, wE),
                                angle_table=inject.histogram_table(eA, wA), bins=True)
    inj(batch=3)
    torch.cuda.synchronize()
    n = p.n_per_batch
    i = np.arange(n, dtype=np.uint64)
    ctr = np.stack([i & 0xFFFFFFFF, np.full(n, 3), np.zeros(n), i >> 32], axis=1)
    c = inject.philox4x32_10(ctr, (11, 0)).astype(np.float64)
    u = (c + 0.5) * 2.0 ** -32
    for w, col, got in ((wE, 1, inj.bin_e), (wA, 2, inj.bin_a)):
        cdf = inject.histogram_table(np.arange(len(w) + 1.0), w)[1]
        want = np.clip(np.searchsorted(cdf, u[:, col], side="right") - 1, 0, len(w) - 1)
        np.testing.assert_array_equal(got.cpu().numpy().astype(np.int64), want)


def test_tally_equals_bincount_of_the_particles(mods):
    torch, adjoint, _, _ = mods
    case, rec, hist = record(mods, n=1 << 14, batches=1, k=1)
    n = case.p.n_per_batch
    st = case.status[:2 * n].cpu().numpy()
    hit = case.hit[:2 * n].cpu().numpy()
    slot = rec.slot.cpu().numpy()
    be, ba = rec.injector.bin_e.cpu().numpy().astype(int), rec.injector.bin_a.cpu().numpy().astype(int)
    ne, na, m = hist.ne, hist.na, case.m
    want = np.zeros((ne + na + 2, m), np.int64)
    ion = np.flatnonzero(st[:n] == 1)
    el = np.flatnonzero(st[n:] == 1)
    s_i, s_e = slot[hit[ion]], slot[hit[n + el]]
    assert (s_i >= 0).all() and (s_e >= 0).all()
    np.add.at(want, (be[ion], s_i), 1)
    np.add.at(want, (ne + ba[ion], s_i), 1)
    np.add.at(want, (ne + na, s_i), 1)
    np.add.at(want, (ne + na + 1, s_e), 1)
    np.testing.assert_array_equal(hist.tables()[0], want)


def test_replay_at_unit_weights_is_the_traced_run(mods, recorded):
    torch, adjoint, _, _ = mods
    case, rec, hist = recorded
    out = adjoint.objectives(hist)
    rho = case.rho_s.cpu().numpy()
    np.testing.assert_allclose(out["rho"].detach().cpu().numpy(), rho, rtol=0, atol=1e-12 * np.abs(rho).max())
    h = case.history()
    np.testing.assert_array_equal(out["ratio_i_bottom"].detach().cpu().numpy(), h["ratio_i_bottom"])
    np.testing.assert_allclose(out["phi_bottom"].item(), h["bottom center"][-1], rtol=1e-9)


MODES = {"floating": {}, "dielectric": dict(mask_type="dielectric"),
         "driven": dict(field_mode="fixed", substrate_voltage=-20.0, mask_voltage=-10.0)}


@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("modes", [0, 4])
def test_reverse_sweep_matches_the_fp64_torch_gradient(mods, mode, modes):
    """Floating conductor, dielectric mask (no conductor) and driven conductor, with and
    without the field-feedback term: the CUDA reverse sweep against torch.autograd of
    the FP64 oracle."""
    torch, adjoint, _, _ = mods
    case, rec, hist = record(mods, n=1 << 14, batches=8, k=3, modes=modes, **MODES[mode])
    dev = case.dev
    f64 = torch.float64
    rE = torch.ones(hist.ne, dtype=f64, device=dev, requires_grad=True)
    rA = torch.ones(hist.na, dtype=f64, device=dev, requires_grad=True)
    rho0 = hist.rho0.clone().requires_grad_(True)
    rho, bottom = adjoint.SurfaceCharge.apply(rE, rA, rho0, hist, hist.has_feedback)
    g_row = case.G[probe_row(case)[0]].to(f64)
    norm = case._desc.bottom_norm
    J = (g_row * rho).sum() + bottom[-1] / norm + 0.1 * bottom[:-1].sum() / norm
    J.backward()
    sur = oracle_of(case)
    oE = torch.ones(hist.ne, dtype=f64, requires_grad=True)
    oA = torch.ones(hist.na, dtype=f64, requires_grad=True)
    o0 = hist.rho0.cpu().clone().requires_grad_(True)
    fb = tuple(t.cpu() for t in hist.feedback_arrays()) if hist.has_feedback else None
    orho, obottom = sur.run(hist.tables(), hist.ne, hist.na, oE, oA, o0, feedback=fb)
    oJ = (g_row.cpu() * orho).sum() + obottom[-1] / norm + 0.1 * obottom[:-1].sum() / norm
    oJ.backward()
    for got, want in ((rE.grad, oE.grad), (rA.grad, oA.grad), (rho0.grad, o0.grad)):
        got, want = got.cpu().numpy(), want.numpy()
        np.testing.assert_allclose(got, want, rtol=1e-8, atol=1e-11 * np.abs(want).max())


def test_adjoint_poisson_solve_is_the_green_row(mods, recorded):
    """The backward of the probe potential (one FP64 adjoint solve) equals the
    probe's row of the surface Green's operator."""
    torch, adjoint, _, _ = mods
    case, rec, hist = recorded
    rho = case.rho_s.clone().requires_grad_(True)
    row, cell = probe_row(case)
    phi = adjoint.ProbePotential.apply(rho, case, [cell])[0]
    phi.backward()
    want = case.G[row].double().cpu().numpy()
    np.testing.assert_allclose(rho.grad.cpu().numpy(), want, rtol=1e-9, atol=1e-9 * np.abs(want).max())


def gradients(mods, hist, feedback=None):
    torch, adjoint, _, _ = mods
    dev, f64 = hist.case.dev, torch.float64
    wE = torch.tensor(hist.energy_weights, dtype=f64, device=dev, requires_grad=True)
    wA = torch.tensor(hist.angle_weights, dtype=f64, device=dev, requires_grad=True)
    out = adjoint.objectives(hist, wE, wA, feedback=feedback)
    J = out["phi_bottom"] + 10.0 * out["ratio_i_bottom"][-1]
    J.backward()
    return wE.grad.cpu().numpy(), wA.grad.cpu().numpy()


def test_gradient_matches_central_differences_per_bin(mods, recorded):
    """Relative step 1e-3 on each bin weight, central differences of the same
    objective over the stored histories: agreement to 1e-3 relative."""
    torch, adjoint, _, _ = mods
    case, rec, hist = recorded
    gE, gA = gradients(mods, hist)
    dev, f64 = case.dev, torch.float64
    h = 1e-3

    def J(wE, wA):
        with torch.no_grad():
            out = adjoint.objectives(hist, torch.tensor(wE, dtype=f64, device=dev),
                                     torch.tensor(wA, dtype=f64, device=dev))
            return out["phi_bottom"].item() + 10.0 * out["ratio_i_bottom"][-1].item()

    for w0, g, which in ((hist.energy_weights, gE, 0), (hist.angle_weights, gA, 1)):
        fd = np.empty_like(g)
        for j in range(len(w0)):
            wp, wm = w0.copy(), w0.copy()
            wp[j] *= 1 + h
            wm[j] *= 1 - h
            args_p = (wp, hist.angle_weights) if which == 0 else (hist.energy_weights, wp)
            args_m = (wm, hist.angle_weights) if which == 0 else (hist.energy_weights, wm)
            fd[j] = (J(*args_p) - J(*args_m)) / (2 * h * w0[j])
        np.testing.assert_allclose(g, fd, rtol=1e-3, atol=1e-3 * np.abs(g).max())


def test_gradient_is_scale_invariant(mods, recorded):
    """The objectives depend on the weights only through the normalised bin
    probabilities, so the gradient is orthogonal to the weights."""
    case, rec, hist = recorded
    gE, gA = gradients(mods, hist)
    assert abs(np.dot(gE, hist.energy_weights)) <= 1e-9 * np.abs(gE).max() * hist.energy_weights.sum()
    assert abs(np.dot(gA, hist.angle_weights)) <= 1e-9 * np.abs(gA).max() * hist.angle_weights.sum()


def test_checkpoint_chunks_and_npz_roundtrip_change_nothing(mods, recorded, tmp_path):
    torch, adjoint, _, _ = mods
    case, rec, hist = recorded
    case2, rec2, hist2 = record(mods, k=12)   # one chunk instead of 5 + 5 + 2
    np.testing.assert_array_equal(hist2.tables(), hist.tables())
    hist.save(tmp_path / "h.npz")
    hist3 = adjoint.History.load(tmp_path / "h.npz", case)
    assert [len(c) for c in hist3.chunks] == [5, 5, 2]
    g1, g3 = gradients(mods, hist), gradients(mods, hist3)
    np.testing.assert_array_equal(g1[0], g3[0])
    np.testing.assert_array_equal(g1[1], g3[1])


def test_feedback_recording_leaves_the_run_unchanged(mods, recorded, recorded_fb):
    """Measuring the responses at the checkpoints traces extra copies of the batch
    but restores the charge and field: the recorded run and its tables are the plain
    run's."""
    case, _, hist = recorded
    case_fb, _, hist_fb = recorded_fb
    np.testing.assert_array_equal(hist_fb.tables(), hist.tables())
    np.testing.assert_array_equal(case_fb.rho_s.cpu().numpy(), case.rho_s.cpu().numpy())
    assert hist_fb.resp_index == [0] * 5 + [1] * 5 + [2] * 2


def test_reverse_sweep_with_feedback_matches_the_fp64_torch_gradient(mods, recorded_fb, tmp_path):
    torch, adjoint, _, _ = mods
    case, rec, hist = recorded_fb
    f64 = torch.float64
    wE = torch.tensor(hist.energy_weights, dtype=f64, device=case.dev, requires_grad=True)
    wA = torch.tensor(hist.angle_weights, dtype=f64, device=case.dev, requires_grad=True)
    rho0 = hist.rho0.clone().requires_grad_(True)
    out = adjoint.objectives(hist, wE, wA, rho0)
    assert hist.has_feedback
    norm = case._desc.bottom_norm
    J = out["phi_bottom"] + 10.0 * out["ratio_i_bottom"][-1] + out["ratio_i_bottom"][:-1].sum()
    J.backward()
    sur = oracle_of(case)
    row, cell = probe_row(case)
    g_row = case.G[row].to(f64).cpu()
    ext = case.t_ext[cell].item()
    fb = tuple(t.cpu() for t in hist.feedback_arrays())
    owE = torch.tensor(hist.energy_weights, dtype=f64, requires_grad=True)
    owA = torch.tensor(hist.angle_weights, dtype=f64, requires_grad=True)
    o0 = hist.rho0.cpu().clone().requires_grad_(True)
    rE = (owE / owE.sum()) / torch.tensor(hist.energy_weights / hist.energy_weights.sum())
    rA = (owA / owA.sum()) / torch.tensor(hist.angle_weights / hist.angle_weights.sum())
    orho, obottom = sur.run(hist.tables(), hist.ne, hist.na, rE, rA, o0, feedback=fb)
    oJ = ext + (g_row * orho).sum() + 10.0 * obottom[-1] / norm + obottom[:-1].sum() / norm
    oJ.backward()
    for got, want in ((wE.grad, owE.grad), (wA.grad, owA.grad), (rho0.grad, o0.grad)):
        got, want = got.cpu().numpy(), want.numpy()
        np.testing.assert_allclose(got, want, rtol=1e-8, atol=1e-10 * np.abs(want).max())
    # the responses change the gradient, and survive the NPZ round trip
    g_plain = gradients(mods, hist, feedback=False)
    g_fb = gradients(mods, hist)
    assert np.abs(g_fb[0] - g_plain[0]).max() > 1e-6 * np.abs(g_plain[0]).max()
    hist.save(tmp_path / "fb.npz")
    g_rt = gradients(mods, adjoint.History.load(tmp_path / "fb.npz", case))
    np.testing.assert_array_equal(g_rt[0], g_fb[0])
    np.testing.assert_array_equal(g_rt[1], g_fb[1])


def test_gradient_tracks_the_full_charging_chain(mods):
    """AR-5 workload at full size (2^20 ions + 2^20 electrons per batch, 50 batches):
    directional derivatives of the adjoint (32 feedback modes measured every batch)
    against central differences of the full charging chain, each chain re-traced
    with the perturbed histograms on the same Philox draws (common random numbers),
    steps of +-10% on the 140 eV peak's bins and on the angle bins above 3 deg.

    Both are Monte Carlo estimates: the chain's derivative over 6 seeds and the adjoint
    over 3 recorded runs give means and standard errors, and the two means must agree
    within 3 combined standard errors, for the bottom-centre potential and the bottom
    ion flux.  The chain is nonlinear in the weights, so a central difference carries a
    truncation error of order h^2 (about 1 % at h = 0.1 on the angle direction); the
    chain's derivative is therefore the Richardson extrapolation (4 D(h/2) - D(h)) / 3
    of the differences at h = 0.1 and 0.05 on the same draws.  Its relative standard
    error (the floor under any comparison at this sample size) is printed; without the
    feedback term the potential's error is larger than with it."""
    torch, adjoint, inject, ChargingCase = mods
    p, eE, wE, eA, wA = adjoint.adjoint_workload()
    B = p.n_batches
    f64 = torch.float64
    cE = 0.5 * (eE[1:] + eE[:-1])
    cA = np.degrees(0.5 * (eA[1:] + eA[:-1]))
    directions = ((np.where(np.abs(cE - 140) < 15, 1.0, 0.0), np.zeros_like(wA)),
                  (np.zeros_like(wE), np.where(cA > 3, 1.0, 0.0)))

    def adjoint_derivatives(seed):
        case = ChargingCase(p, precision="f32", max_batches=B)
        hist = adjoint.AdjointRecorder(case, eE, wE, eA, wA, seed=seed).run(B)
        out = {}
        for fb in (True, False):
            for name in ("phi", "flux"):
                gE = torch.tensor(wE, dtype=f64, device=case.dev, requires_grad=True)
                gA = torch.tensor(wA, dtype=f64, device=case.dev, requires_grad=True)
                o = adjoint.objectives(hist, gE, gA, feedback=fb)
                (o["phi_bottom"] if name == "phi" else o["ratio_i_bottom"][-1]).backward()
                g = (gE.grad.cpu().numpy(), gA.grad.cpu().numpy())
                out[fb, name] = [float(np.dot(g[0], wE * vE) + np.dot(g[1], wA * vA)) for vE, vA in directions]
        return out

    def chain(wE_, wA_, seed):
        c = ChargingCase(p, precision="f32", max_batches=B)
        inj = inject.DeviceInjector(c, seed, energy_table=inject.histogram_table(eE, wE_),
                                    angle_table=inject.histogram_table(eA, wA_))
        for _ in range(B):
            inj()
            c.step()
        h = c.history()
        return np.array([h["bottom center"][-1], h["ratio_i_bottom"][-1]])

    adj = [adjoint_derivatives(s) for s in (21, 31, 41)]

    def central(vE, vA, h, seed):
        return (chain(wE * (1 + h * vE), wA * (1 + h * vA), seed) - chain(wE * (1 - h * vE), wA * (1 - h * vA), seed)) \
            / (2 * h)

    for d, (vE, vA) in enumerate(directions):
        coarse = np.array([central(vE, vA, 0.1, s) for s in range(21, 27)])
        fine = np.array([central(vE, vA, 0.05, s) for s in range(21, 27)])
        fd = (4 * fine - coarse) / 3
        fd_mean, fd_se = fd.mean(axis=0), fd.std(axis=0, ddof=1) / np.sqrt(len(fd))
        print(f"direction {d}: central differences h=0.1 {coarse.mean(axis=0)}, h=0.05 {fine.mean(axis=0)}")
        for j, name in enumerate(("phi", "flux")):
            a = np.array([r[True, name][d] for r in adj])
            a_mean, a_se = a.mean(), a.std(ddof=1) / np.sqrt(len(a))
            print(f"direction {d} {name}: adjoint {a_mean:.6g} +- {a_se:.2g}, chain {fd_mean[j]:.6g} +- {fd_se[j]:.2g} "
                  f"(chain relative standard error {fd_se[j] / abs(fd_mean[j]):.2%})")
            assert abs(a_mean - fd_mean[j]) <= 3 * np.hypot(a_se, fd_se[j]), (name, d, a, fd[:, j])
        frozen = np.mean([r[False, "phi"][d] for r in adj])
        assert abs(frozen - fd_mean[0]) > abs(np.mean([r[True, "phi"][d] for r in adj]) - fd_mean[0])
