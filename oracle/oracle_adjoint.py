"""ORACLE -- test infrastructure only (the checker, never the product).

FP64 PyTorch restatement of the adjoint's surrogate recurrence, written with
plain differentiable torch operations so that torch.autograd gives the reference
gradient the hand-written reverse sweep (tb_adjoint.cu) is checked against.

The surrogate is the reference's per-batch charge update
(trench_charging_2d.py:1239-1266, restated over the whole grid in
oracle_fields.BatchState.step) on the surface-cell vector, driven by ion deposits
reweighted from stored tally tables:

    ci_b = Ni_b + (rE - 1) . TE_b + (rA - 1) . TA_b,   ce_b = electron deposit,

table rows [0, ne) ions by energy bin, [ne, ne + na) ions by angle bin, ne + na all
ions, ne + na + 1 electrons.  The reference has no gradient; at r = 1 this
recurrence is checked against BatchState (which is pinned to reference runs), and
its autograd gradient against central finite differences of itself.
"""
import numpy as np
import torch

SFLAG_COND, SFLAG_BOTTOM = 1, 4


def conductor_step(n_i, n_e, q, C, Te, drift):
    """trench_charging_2d.py:815-830 on torch scalars."""
    x_i = q * n_i / C + drift
    x_e = q * n_e / C
    if float(n_e.detach() if torch.is_tensor(n_e) else n_e) == 0:
        return x_i
    k = x_i / Te
    frac = -torch.expm1(-k) / k if float(k.detach()) != 0 else torch.ones_like(k)
    return -Te * torch.logaddexp(-k, torch.log(x_e / Te * frac))


class Surrogate:
    """Charge update of one case on the surface vector (m slots, FP64).

    sflag: (m,) bits 1 = conductor, 4 = bottom; leak_M: (m, m) implicit leakage
    operator or None; leak_h: (m,) dt G phi_ext or None; g_s: (m,) floating-conductor
    response or None; c_slot: slot holding the conductor's charge."""

    def __init__(self, sflag, leak_M, leak_h, g_s, c_slot, floating, driven, q, dx, C, Te):
        f64 = torch.float64
        t = lambda a: None if a is None else torch.as_tensor(np.asarray(a), dtype=f64)
        sflag = np.asarray(sflag)
        self.cond = torch.as_tensor((sflag & SFLAG_COND) != 0)
        self.bottom = torch.as_tensor((sflag & SFLAG_BOTTOM) != 0)
        self.M, self.h, self.g = t(leak_M), t(leak_h), t(g_s)
        self.c_slot = int(c_slot)
        self.floating, self.driven = bool(floating), bool(driven)
        self.q, self.dx, self.C, self.Te = float(q), float(dx), float(C), float(Te)

    def run(self, tables, ne, na, rE, rA, rho0, feedback=None):
        """tables (B, ne + na + 2, m) integers; rE (ne,), rA (na,), rho0 (m,) FP64
        tensors.  Returns (rho after the last batch, bottom ion deposit per batch).
        feedback = (basis (m, K), resp_i (sets, m, K), resp_e, index (B,)): the
        deposits' linear response to the charge state along the basis, entering as
        resp (basis^T (rho - rho.detach())) -- zero in value, present in the gradient."""
        T_all = torch.as_tensor(np.asarray(tables), dtype=torch.float64)
        dx2 = self.dx * self.dx
        rho = rho0
        bottom = []
        for b, T in enumerate(T_all):
            ci = T[ne + na] + (rE - 1.0) @ T[:ne] + (rA - 1.0) @ T[ne:ne + na]
            ce = T[ne + na + 1]
            if feedback is not None and int(feedback[3][b]) >= 0:
                V, Ri, Re, index = feedback
                coef = V.T @ (rho - rho.detach())
                ci = ci + Ri[int(index[b])] @ coef
                ce = ce + Re[int(index[b])] @ coef
            drho = torch.where(self.cond, torch.zeros_like(ci), (ci - ce) * self.q / dx2)
            r = rho + drho
            if self.M is not None:
                w = r * dx2 + (self.h if self.h is not None else 0.0)
                r = (self.M @ w) / dx2
            if self.driven:
                r = torch.where(self.cond, torch.zeros_like(r), r)
            if self.floating and self.c_slot >= 0:
                drift = ((r - rho) * self.g).sum() * dx2
                dV = conductor_step(ci[self.cond].sum(), ce[self.cond].sum(), self.q, self.C, self.Te, drift)
                bump = torch.zeros_like(r)
                bump[self.c_slot] = 1.0
                r = r + bump * (self.C * (dV - drift) / dx2)
            rho = r
            bottom.append(ci[self.bottom].sum())
        return rho, torch.stack(bottom)
