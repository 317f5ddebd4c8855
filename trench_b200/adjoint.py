"""Adjoint of the charging loop: gradients of charging objectives with respect to
the ion energy/angle histogram weights and the surface-charge vector.

The reference has no gradient; this module has no counterpart there.  The
objectives are those of the reference's history (trench_charging_2d.py:1163,
1273-1276): the potential of the "bottom center" probe after the last batch and
the bottom ion-flux ratio of each batch.

Method.  Ions are drawn from histogram tables (energy bins, polar-angle bins);
the gradient with respect to the bin weights is taken by likelihood-ratio
reweighting of the traced histories.  ``AdjointRecorder`` runs a ChargingCase
forward with device injection from the tables and records, per batch, the
absorbed ions tallied by (table bin, surface slot) and the electrons by slot
(``tb_tally``); every ``checkpoint_every`` batches the tallies move to pinned host
memory (and, if asked, to an NPZ file), so the device holds one chunk of them.
``SurfaceCharge`` replays the charge update over the stored histories with each
ion reweighted by its bins' probability ratios r (the trajectories held fixed)
and returns the final surface charge and the per-batch bottom ion deposit; its
backward is the reverse sweep of that recurrence (``tb_adjoint_reverse``).
``ProbePotential`` evaluates the potential at grid cells from a surface charge;
its backward is one FP64 adjoint Poisson solve (the discrete operator, with the
floating conductor as one unknown, is symmetric, so the adjoint solve is a solve).
At r = 1 the replay reproduces the traced run's surface charge.

Field feedback.  Holding the trajectories fixed misses how a changed charge bends
later trajectories, which damps the real response.  With ``feedback_modes=K`` the
recorder also measures, at every checkpoint, the ion and electron deposits'
linear response to the charge state along K surface-charge modes -- the leading
right singular vectors of the surface Green's operator on the vacuum cells, i.e.
the charge patterns that move the potential the particles see the most -- by
central differences on the same injected particles (common random numbers), each
mode scaled to move the vacuum potential by at most ``feedback_volts``, every
``feedback_every`` batches.  The reverse sweep adds that response (a rank-K
linearisation of the field's effect, held between measurements).  On the AR-5
workload (2^20 ions per batch, 50 batches, 3 recorded runs against 8 chain seeds)
the response measured every batch brings both gradients (bottom-centre potential,
bottom ion flux, along the 140 eV energy bins and along the angle bins above 3 deg)
within the chain derivative's own standard error (0.1-0.3 % for the potential); a
response held for 5 batches leaves a 0.8 % bias along the angle bins, 64 modes
instead of 32 do not remove it, and without the feedback the errors are 4-100 %.
"""
import ctypes

import numpy as np
import torch

from . import _capi
from .inject import DeviceInjector, histogram_table
from .params import EPS0
from .tracer import _ptr


class History:
    """Stored traced histories of one recorded run: per batch an int32 table
    (n_energy + n_angle + 2, m) -- ions by energy bin, ions by angle bin, all ions,
    electrons -- by surface slot; in chunks of ``checkpoint_every`` batches in
    pinned host memory."""

    def __init__(self, case, energy, angle, seed, checkpoint_every, rho0, start_batch):
        self.case = case
        self.energy_edges, self.energy_weights = (np.asarray(v, dtype=np.float64) for v in energy)
        self.angle_edges, self.angle_weights = (np.asarray(v, dtype=np.float64) for v in angle)
        self.ne, self.na = len(self.energy_weights), len(self.angle_weights)
        self.rows = self.ne + self.na + 2
        self.seed = int(seed)
        self.checkpoint_every = int(checkpoint_every)
        self.rho0 = rho0
        self.start_batch = int(start_batch)
        self.chunks = []
        self._leak_MT = None
        # field feedback: basis (m, K) and per-chunk responses (m, K) of ions and electrons
        self.basis = None
        self.resp_i, self.resp_e = [], []
        self.resp_index = []          # per batch: response set or -1

    @property
    def n_batches(self):
        return sum(len(c) for c in self.chunks)

    @property
    def has_feedback(self):
        return self.basis is not None and len(self.resp_i) > 0

    def tables(self):
        """All batches' tables as one host array (n_batches, rows, m)."""
        return torch.cat(self.chunks).numpy() if self.chunks else np.zeros((0, self.rows, self.case.m), np.int32)

    def leak_MT(self):
        if self._leak_MT is None and self.case.leak_M is not None:
            self._leak_MT = self.case.leak_M.T.contiguous()
        return self._leak_MT

    def feedback_arrays(self):
        """(basis (m, K), resp_i (sets, m, K), resp_e, resp_index (n_batches,)) on the device."""
        dev = self.case.dev
        return (self.basis.contiguous(), torch.stack(self.resp_i).contiguous(), torch.stack(self.resp_e).contiguous(),
                torch.tensor(self.resp_index, dtype=torch.int32, device=dev))

    def save(self, path):
        """The histories and what the replay needs of the run, pickle-free."""
        extra = {}
        if self.has_feedback:
            b, ri, re, ix = self.feedback_arrays()
            extra = dict(basis=b.cpu().numpy(), resp_i=ri.cpu().numpy(), resp_e=re.cpu().numpy(),
                         resp_index=ix.cpu().numpy())
        np.savez(path, energy_edges=self.energy_edges, energy_weights=self.energy_weights,
                 angle_edges=self.angle_edges, angle_weights=self.angle_weights,
                 seed=np.array(self.seed), checkpoint_every=np.array(self.checkpoint_every),
                 start_batch=np.array(self.start_batch), rho0=self.rho0.cpu().numpy(), tables=self.tables(),
                 **extra)

    @staticmethod
    def load(path, case):
        with np.load(path, allow_pickle=False) as z:
            h = History(case, (z["energy_edges"], z["energy_weights"]), (z["angle_edges"], z["angle_weights"]),
                        int(z["seed"]), int(z["checkpoint_every"]),
                        torch.from_numpy(z["rho0"]).to(case.dev), int(z["start_batch"]))
            t = z["tables"]
            if "basis" in z:
                dev = case.dev
                h.basis = torch.from_numpy(z["basis"]).to(dev)
                h.resp_i = list(torch.from_numpy(z["resp_i"]).to(dev))
                h.resp_e = list(torch.from_numpy(z["resp_e"]).to(dev))
                h.resp_index = [int(v) for v in z["resp_index"]]
        if t.ndim != 3 or t.shape[1:] != (h.rows, case.m):
            raise ValueError("the stored tables do not fit this case")
        k = h.checkpoint_every
        h.chunks = [torch.from_numpy(t[i:i + k].copy()).pin_memory() for i in range(0, len(t), k)]
        return h


class AdjointRecorder:
    """Runs `case` forward with ions from histogram tables (edges and weights of the
    energy bins in eV and of the polar-angle bins in radians, the angle's sign drawn
    at random) and electrons as in the reference, recording the histories.
    feedback_modes=0 records no field feedback (the pure likelihood-ratio gradient,
    one forward pass); the default, 32 modes measured every batch, costs 2 x 32 extra
    traces of a batch per batch."""

    def __init__(self, case, energy_edges, energy_weights, angle_edges, angle_weights, seed=0,
                 angle_random_sign=True, checkpoint_every=10, feedback_modes=32, feedback_volts=0.5,
                 feedback_every=1):
        if case.rf is not None:
            raise ValueError("the adjoint covers DC charging; circuit_rf is not supported")
        if int(checkpoint_every) < 1 or int(feedback_every) < 1:
            raise ValueError("checkpoint_every and feedback_every must be at least 1")
        self.case = case
        self.energy = histogram_table(energy_edges, energy_weights)[0], np.asarray(energy_weights, np.float64)
        self.angle = histogram_table(angle_edges, angle_weights)[0], np.asarray(angle_weights, np.float64)
        self.seed = int(seed)
        self.injector = DeviceInjector(case, seed, energy_table=histogram_table(energy_edges, energy_weights),
                                       angle_table=histogram_table(angle_edges, angle_weights),
                                       angle_random_sign=angle_random_sign, bins=True)
        ne, na = len(self.energy[1]), len(self.angle[1])
        self.rows = ne + na + 2
        dev = case.dev
        if case.hit is None:
            case.hit = torch.full((case.capacity,), -1, dtype=torch.int32, device=dev)
        slot = torch.full((case.n,), -1, dtype=torch.int32, device=dev)
        slot[case.t_surf.long()] = torch.arange(case.m, dtype=torch.int32, device=dev)
        self.slot = slot
        self.k = int(checkpoint_every)
        self.chunk = torch.zeros((self.k, self.rows, case.m), dtype=torch.int32, device=dev)
        a = _capi.TallyArgs()
        a.n_species = int(case.p.n_per_batch)
        a.d_status, a.d_hit = _ptr(case.status), _ptr(case.hit)
        a.d_bin_e, a.d_bin_a = _ptr(self.injector.bin_e), _ptr(self.injector.bin_a)
        a.d_slot = _ptr(self.slot)
        a.m, a.n_energy, a.n_angle = case.m, ne, na
        self._targs = a
        self._j = 0
        self.K = int(feedback_modes)
        self.feedback_every = int(feedback_every)
        self.basis = self.eps = None
        if self.K > 0:
            # leading right singular vectors of G on the vacuum rows; each mode scaled to move
            # the vacuum potential by feedback_volts at most
            vac_rows = torch.from_numpy(case.vac.ravel()[case.rows]).to(dev)
            Gv = case.G[vac_rows].to(torch.float64)
            _, _, Vh = torch.linalg.svd(Gv, full_matrices=False)
            self.K = min(self.K, Vh.shape[0])
            self.basis = Vh[:self.K].T.contiguous()
            self.eps = float(feedback_volts) / (Gv @ self.basis).abs().amax(dim=0)

    def _tally(self):
        case = self.case
        self._targs.d_table = _ptr(self.chunk[self._j])
        s = ctypes.c_void_p(torch.cuda.current_stream(case.dev).cuda_stream)
        case.ctx.check(_capi.lib().tb_tally(case.ctx.handle, ctypes.byref(self._targs), s))

    def _responses(self):
        """Ion and electron deposit per unit charge along each mode at the current state,
        central differences on the loaded particles (the field is restored after)."""
        case = self.case
        S = case.t_surf.long()
        n = case.n_loaded
        rho = case.rho_s.clone()
        Ui = torch.zeros((case.m, self.K), dtype=torch.float64, device=case.dev)
        Ue = torch.zeros_like(Ui)
        for j in range(self.K):
            out = []
            for sgn in (1.0, -1.0):
                case.rho_s.copy_(rho + sgn * self.eps[j] * self.basis[:, j])
                case._potential()
                case._trace_only(n)
                out.append((case.counts[0][S].to(torch.float64), case.counts[1][S].to(torch.float64)))
            Ui[:, j] = (out[0][0] - out[1][0]) / (2 * self.eps[j])
            Ue[:, j] = (out[0][1] - out[1][1]) / (2 * self.eps[j])
        case.rho_s.copy_(rho)
        case._potential()
        return Ui, Ue

    def run(self, n_batches, path=None):
        """Trace `n_batches` batches from the case's current state; returns the History.
        With `path`, the histories so far are written there at every checkpoint."""
        case = self.case
        n_batches = int(n_batches)
        with torch.cuda.device(case.dev):
            hist = History(case, self.energy, self.angle, self.seed, self.k, case.rho_s.clone(),
                           case.batches_done())
            hist.basis = self.basis
            try:
                for b in range(n_batches):
                    j = self._j = b % self.k
                    self.chunk[j].zero_()
                    self.injector()
                    if self.K > 0:
                        if b % self.feedback_every == 0:
                            Ui, Ue = self._responses()
                            hist.resp_i.append(Ui)
                            hist.resp_e.append(Ue)
                        hist.resp_index.append(len(hist.resp_i) - 1)
                    case.after_trace = self._tally
                    case.step()
                    case.after_trace = None
                    if j == self.k - 1 or b == n_batches - 1:
                        host = torch.empty((j + 1, self.rows, case.m), dtype=torch.int32, pin_memory=True)
                        host.copy_(self.chunk[:j + 1], non_blocking=True)
                        hist.chunks.append(host)
                        if path is not None:
                            torch.cuda.current_stream(case.dev).synchronize()
                            hist.save(path)
            finally:
                case.after_trace = None
            torch.cuda.current_stream(case.dev).synchronize()
            case.check()
        return hist


def adjoint_workload(n_per_batch=1 << 20, n_batches=50, seed=3):
    """AR-5 adjoint-sensitivity workload: 60x180 grid, trench 20 cells wide x 100 deep,
    floor 10, conductive (floating) mask 20 cells, 50 vacuum rows; ions from a 64-bin
    energy histogram over 0-300 eV (Gaussians at 40 and 140 eV, sigma 6 eV, equal
    weight, plus 2% spread evenly so every bin is drawn) and a 32-bin polar-angle
    histogram over 0-10 deg (half-Gaussian sigma 3 deg plus the same 2% floor, random
    sign); electrons Maxwellian 3 eV.  Returns (params, energy edges, energy weights,
    angle edges, angle weights)."""
    from dataclasses import replace
    from .params import Params
    p = replace(Params(), nx=60, trench_w=20, trench_d=100, floor_t=10, mask_t=20, n_vac=50,
                mask_type="conductor", field_mode="floating", bias="dc", electron_temp_eV=3.0,
                n_per_batch=int(n_per_batch), n_batches=int(n_batches), seed=int(seed))
    eE = np.linspace(0.0, 300.0, 65)
    cE = 0.5 * (eE[1:] + eE[:-1])
    wE = 0.5 * np.exp(-0.5 * ((cE - 40.0) / 6.0) ** 2) + 0.5 * np.exp(-0.5 * ((cE - 140.0) / 6.0) ** 2)
    wE = 0.98 * wE / wE.sum() + 0.02 / len(wE)
    eA = np.radians(np.linspace(0.0, 10.0, 33))
    cA = 0.5 * (eA[1:] + eA[:-1])
    wA = np.exp(-0.5 * (cA / np.radians(3.0)) ** 2)
    wA = 0.98 * wA / wA.sum() + 0.02 / len(wA)
    return p, eE, wE, eA, wA


def _adjoint_args(hist, T, nb, rE, rA, rho, scal, bottom, MT):
    a = _capi.AdjointArgs()
    a.n_batches, a.n_energy, a.n_angle = nb, hist.ne, hist.na
    a.d_tables = _ptr(T)
    a.d_rE = _ptr(rE) if rE is not None else None
    a.d_rA = _ptr(rA) if rA is not None else None
    a.d_leak_MT = _ptr(MT) if MT is not None else None
    a.d_rho, a.d_scal, a.d_bottom = _ptr(rho), _ptr(scal), _ptr(bottom)
    a.n_basis = 0
    return a


class SurfaceCharge(torch.autograd.Function):
    """(rE, rA, rho0) -> (surface charge after the last batch, bottom ion deposit per
    batch) over the stored histories; backward by the reverse sweep (with the field
    feedback when `feedback` and the history holds it)."""

    @staticmethod
    def forward(ctx, rE, rA, rho0, hist, feedback=False):
        case = hist.case
        dev, f64 = case.dev, torch.float64
        rE = rE.detach().to(dev, f64).contiguous()
        rA = rA.detach().to(dev, f64).contiguous()
        rho = rho0.detach().to(dev, f64).clone().contiguous()
        B = hist.n_batches
        scal = torch.zeros((B, 4), dtype=f64, device=dev)
        bottom = torch.zeros(B, dtype=f64, device=dev)
        L = _capi.lib()
        with torch.cuda.device(dev):
            s = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
            b0 = 0
            for chunk in hist.chunks:
                nb = len(chunk)
                T = chunk.to(dev, non_blocking=True)
                a = _adjoint_args(hist, T, nb, rE, rA, rho, scal[b0:], bottom[b0:], None)
                case.ctx.check(L.tb_adjoint_forward(case.ctx.handle, ctypes.byref(case._desc), ctypes.byref(a), s))
                b0 += nb
        ctx.hist = hist
        ctx.feedback = bool(feedback) and hist.has_feedback
        ctx.save_for_backward(scal)
        return rho, bottom

    @staticmethod
    def backward(ctx, g_rho, g_bottom):
        hist = ctx.hist
        (scal,) = ctx.saved_tensors
        case = hist.case
        dev, f64, m, B = case.dev, torch.float64, case.m, hist.n_batches
        lam = (g_rho.detach().to(dev, f64).clone() if g_rho is not None
               else torch.zeros(m, dtype=f64, device=dev)).contiguous()
        gb = (g_bottom.detach().to(dev, f64) if g_bottom is not None
              else torch.zeros(B, dtype=f64, device=dev)).contiguous()
        grad = torch.zeros(hist.ne + hist.na, dtype=f64, device=dev)
        fb = hist.feedback_arrays() if ctx.feedback else None
        K = fb[0].shape[1] if fb is not None else 0
        scratch = torch.zeros(2 * m + 4 + K, dtype=f64, device=dev)
        rho_unused = torch.zeros(m, dtype=f64, device=dev)
        bottom_unused = torch.zeros(B, dtype=f64, device=dev)
        MT = hist.leak_MT()
        L = _capi.lib()
        with torch.cuda.device(dev):
            s = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
            end = B
            for chunk in reversed(hist.chunks):
                nb = len(chunk)
                b0 = end - nb
                T = chunk.to(dev, non_blocking=True)
                a = _adjoint_args(hist, T, nb, None, None, rho_unused, scal[b0:], bottom_unused[b0:], MT)
                if fb is not None:
                    a.n_basis = K
                    a.d_basis, a.d_resp_i, a.d_resp_e = _ptr(fb[0]), _ptr(fb[1]), _ptr(fb[2])
                    a.d_resp_index = _ptr(fb[3][b0:])
                case.ctx.check(L.tb_adjoint_reverse(case.ctx.handle, ctypes.byref(case._desc), ctypes.byref(a),
                                                    _ptr(lam), _ptr(gb[b0:]), _ptr(grad), _ptr(scratch), s))
                end = b0
        return grad[:hist.ne], grad[hist.ne:], lam, None, None


class ProbePotential(torch.autograd.Function):
    """rho_s (surface charge density per surface slot) -> potential at flat grid
    cells, phi = external + solve(-rho / eps0); backward by the FP64 adjoint solve."""

    @staticmethod
    def forward(ctx, rho_s, case, cells):
        dev, f64 = case.dev, torch.float64
        cells_t = torch.as_tensor(np.asarray(cells, dtype=np.int64), device=dev)
        b = torch.zeros((1, case.n), dtype=f64, device=dev)
        b[0, case.t_surf.long()] = -rho_s.detach().to(dev, f64) / EPS0
        with torch.cuda.device(dev):
            phi = case.solver.solve_rows(b)[0]
        ctx.case, ctx.cells = case, cells_t
        return case.t_ext[cells_t] + phi[cells_t]

    @staticmethod
    def backward(ctx, g):
        case = ctx.case
        c = torch.zeros((1, case.n), dtype=torch.float64, device=case.dev)
        c[0].index_add_(0, ctx.cells, g.detach().to(torch.float64))
        with torch.cuda.device(case.dev):
            psi = case.solver.solve_rows(c)[0]
        return -psi[case.t_surf.long()] / EPS0, None, None


def bin_ratios(w, w0):
    """Probability ratios of histogram bins, (w / sum w) / (w0 / sum w0); 1 where the
    recorded weight is zero (no ion was drawn there)."""
    p = w / w.sum()
    p0 = w0 / w0.sum()
    safe = torch.where(p0 > 0, p0, torch.ones_like(p0))
    return torch.where(p0 > 0, p / safe, torch.ones_like(p))


def objectives(hist, w_energy=None, w_angle=None, rho0=None, feedback=None):
    """Charging objectives over the recorded run, differentiable with respect to the
    energy and angle bin weights (unnormalised) and the initial surface charge
    (feedback: use the recorded field-feedback response in the backward; default:
    whenever it was recorded):
    ``phi_bottom`` = potential of the "bottom center" probe after the last batch (V),
    ``ratio_i_bottom`` = bottom ion-flux ratio per batch (trench_charging_2d.py:1276),
    ``rho`` = surface charge after the last batch."""
    case = hist.case
    dev, f64 = case.dev, torch.float64
    wE0 = torch.as_tensor(hist.energy_weights, dtype=f64, device=dev)
    wA0 = torch.as_tensor(hist.angle_weights, dtype=f64, device=dev)
    w_energy = wE0 if w_energy is None else w_energy
    w_angle = wA0 if w_angle is None else w_angle
    rho0 = hist.rho0 if rho0 is None else rho0
    feedback = hist.has_feedback if feedback is None else bool(feedback)
    rho, bottom = SurfaceCharge.apply(bin_ratios(w_energy, wE0), bin_ratios(w_angle, wA0), rho0, hist, feedback)
    ix, iy = case.probes["bottom center"]
    phi = ProbePotential.apply(rho, case, [ix * case.ny + iy])[0]
    return dict(phi_bottom=phi, ratio_i_bottom=bottom / case._desc.bottom_norm, rho=rho)
