"""Test-only ctypes shim: a torch.autograd.Function whose forward is a recorded GPU rollout
(vbd_solver_step x steps) and whose backward is the library's adjoint (vbd_solver_backward).
Used only to check the adjoint through torch's autograd machinery."""
import numpy as np
import torch


class VBDRollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mu, lam, x0, v0, solver, steps, dt, iterations, gravity, accel, rho, checkpoint, adj_iters):
        solver.set_materials(mu.detach().cpu().numpy(), lam.detach().cpu().numpy())
        solver.set_positions(x0.detach().cpu().numpy())
        solver.set_velocities(v0.detach().cpu().numpy())
        solver.record(checkpoint)
        for _ in range(steps):
            solver.step(dt, iterations, gravity, accel, rho)
        ctx.solver = solver
        ctx.adj_iters = adj_iters
        return torch.from_numpy(solver.get_positions().astype(np.float64))

    @staticmethod
    def backward(ctx, grad_x):
        gx, gv, gm, gl = ctx.solver.backward(grad_x.detach().cpu().numpy(), None, ctx.adj_iters)
        t = lambda a: torch.from_numpy(a.astype(np.float64))  # noqa: E731
        return t(gm), t(gl), t(gx), t(gv), None, None, None, None, None, None, None, None, None
