"""Thin torch.autograd harness over the C-ABI adjoint (test use only).

KineticEnergyAfterSteps(rho0) = J(q_N), q_0 = Taylor-Green state with the
density field rho0 (velocity and pressure fixed), q_N after len(dts) RK
steps with the given time steps.  backward() returns dJ/drho0 from
cs_adjoint_gradient: dJ/drho0 = lambda_0 . dq_0/drho0 with
dq_0/drho0 = (1, u, v, w, |u|^2 / 2).
"""
import torch


def tgv_state(rho, u, p, gamma=1.4):
    """[5 * lmx] conserved state from density rho, velocity u [3, lmx], pressure p."""
    q = torch.empty(5, rho.numel(), dtype=torch.float64, device=rho.device)
    q[0] = rho
    q[1:4] = rho * u
    q[4] = p / (gamma - 1.0) + 0.5 * rho * (u * u).sum(0)
    return q.reshape(-1)


def primitives(q, gamma=1.4):
    q = q.reshape(5, -1)
    rho = q[0]
    u = q[1:4] / rho
    p = (gamma - 1.0) * (q[4] - 0.5 * rho * (u * u).sum(0))
    return rho, u, p


class KineticEnergyAfterSteps(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho0, u, p, solver, adj, dts, every):
        q = tgv_state(rho0, u, p)
        ctx.save_for_backward(rho0, u, p)
        ctx.adj, ctx.dts, ctx.every = adj, dts, every
        qr = q.clone()
        for dt in dts:
            solver.step(qr, dt)
        return torch.tensor(adj.kinetic_energy(qr), dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        rho0, u, p = ctx.saved_tensors
        q0 = tgv_state(rho0, u, p)
        lam = torch.empty_like(q0)
        ctx.adj.gradient(q0, ctx.dts, ctx.every, lam)
        lam = lam.reshape(5, -1)
        g = lam[0] + (lam[1:4] * u).sum(0) + 0.5 * lam[4] * (u * u).sum(0)
        return gJ.to(g.device) * g, None, None, None, None, None, None
