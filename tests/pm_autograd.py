"""torch.autograd.Function over the C ABI's steps and their adjoints (FP64,
and FP32 with split positions).

Differentiable PM run: particles on the lattice q are displaced by psi (one
3-vector per particle, cell units) with velocities vel_factor * psi, advanced
by `steps` leapfrog KDK steps (steps + 1 force evaluations, half kicks merged),
and scored by the mean squared difference between the final CIC density and a
target density.  backward() runs the hand-written adjoints
(pm_adjoint_deposit_f64, pm_step_adjoint_f64) in reverse, recomputing the
trajectory segment by segment from checkpoints stored every `ckpt` steps, so
only ceil(steps / ckpt) + ckpt particle states are ever held.
"""
import torch


def kdk_schedule(steps, dt):
    """(c_kick, dt_drift) of each of the steps + 1 merged KDK force steps."""
    return [(0.5 * dt if s in (0, steps) else dt, dt if s < steps else 0.0) for s in range(steps + 1)]


def wrap(x, ng):
    return torch.remainder(x, float(ng))


class PMLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, psi, q, plan, ng, mass, c_poisson, dt, steps, target, vel_factor, ckpt):
        sched = kdk_schedule(steps, dt)
        x = [wrap(q[a] + psi[a], ng).contiguous() for a in range(3)]
        v = [(vel_factor * psi[a]).contiguous() for a in range(3)]
        ckpts = {}
        for s, (ck, dd) in enumerate(sched[:-1]):  # the closing half kick does not move particles
            if s % ckpt == 0:
                ckpts[s] = ([t.clone() for t in x], [t.clone() for t in v])
            plan.step(*x, *v, mass, c_poisson, ck, dd)
        delta = plan.deposit(*x, mass)
        n = ng
        diff = delta[:, :, :n] - target
        loss = (diff * diff).mean()
        ctx.save_for_backward(psi)
        ctx.plan, ctx.ng, ctx.mass, ctx.cp, ctx.sched, ctx.ckpts = plan, ng, mass, c_poisson, sched, ckpts
        ctx.x_final, ctx.diff, ctx.vel_factor, ctx.ckpt = x, diff, vel_factor, ckpt
        return loss

    @staticmethod
    def backward(ctx, gloss):
        plan, ng, mass, cp, sched = ctx.plan, ctx.ng, ctx.mass, ctx.cp, ctx.sched
        n = ng
        dbar = torch.zeros((n, n, n + 2), dtype=torch.float64, device=gloss.device)
        dbar[:, :, :n] = ctx.diff * (2.0 / n ** 3) * gloss
        xb = [torch.zeros_like(ctx.x_final[0]) for _ in range(3)]
        vb = [torch.zeros_like(ctx.x_final[0]) for _ in range(3)]
        plan.adjoint_deposit(*ctx.x_final, mass, dbar, xb)
        nsteps = len(sched) - 1
        starts = sorted(ctx.ckpts)
        for a in reversed(starts):
            b = min(a + ctx.ckpt, nsteps)
            x = [t.clone() for t in ctx.ckpts[a][0]]
            v = [t.clone() for t in ctx.ckpts[a][1]]
            states = []
            for s in range(a, b):  # recompute the segment, keeping each step's start positions
                states.append([t.clone() for t in x])
                ck, dd = sched[s]
                plan.step(*x, *v, mass, cp, ck, dd)
            for s in reversed(range(a, b)):
                ck, dd = sched[s]
                plan.step_adjoint(*states[s - a], mass, cp, ck, dd, xb, vb)
        grad = torch.stack([xb[a] + ctx.vel_factor * vb[a] for a in range(3)])
        return grad, None, None, None, None, None, None, None, None, None, None


def loss_fn(psi, q, plan, ng, mass, c_poisson, dt, steps, target, vel_factor=1.0, ckpt=8):
    return PMLoss.apply(psi, q, plan, ng, mass, c_poisson, dt, steps, target, vel_factor, ckpt)


class PMLossSplit(torch.autograd.Function):
    """The same differentiable run on the FP32 split-position path
    (pm_step_f32, pm_adjoint_deposit_f32, pm_step_adjoint_f32).  psi, q and
    the target are FP64 tensors; the state, the mesh and the adjoint arrays
    are FP32, the loss and the returned gradient FP64."""

    @staticmethod
    def forward(ctx, psi, q, plan, ng, mass, c_poisson, dt, steps, target, vel_factor, ckpt):
        sched = kdk_schedule(steps, dt)
        cell, off = plan.split(*[wrap(q[a] + psi[a], ng).contiguous() for a in range(3)])
        v = [(vel_factor * psi[a]).float().contiguous() for a in range(3)]
        ckpts = {}
        for s, (ck, dd) in enumerate(sched[:-1]):
            if s % ckpt == 0:
                ckpts[s] = (cell.clone(), [t.clone() for t in off], [t.clone() for t in v])
            plan.step_split(cell, off, v, mass, c_poisson, ck, dd)
        delta = plan.deposit_split(cell, off, mass)
        diff = delta[:, :, :ng].double() - target
        loss = (diff * diff).mean()
        ctx.save_for_backward(psi)
        ctx.plan, ctx.ng, ctx.mass, ctx.cp, ctx.sched, ctx.ckpts = plan, ng, mass, c_poisson, sched, ckpts
        ctx.final, ctx.diff, ctx.vel_factor, ctx.ckpt = (cell, off), diff, vel_factor, ckpt
        return loss

    @staticmethod
    def backward(ctx, gloss):
        plan, n, mass, cp, sched = ctx.plan, ctx.ng, ctx.mass, ctx.cp, ctx.sched
        cell, off = ctx.final
        dbar = torch.zeros((n, n, n + 2), dtype=torch.float32, device=gloss.device)
        dbar[:, :, :n] = (ctx.diff * (2.0 / n ** 3) * gloss).float()
        xb = [torch.zeros_like(off[0]) for _ in range(3)]
        vb = [torch.zeros_like(off[0]) for _ in range(3)]
        plan.adjoint_deposit_split(cell, off, mass, dbar, xb)
        nsteps = len(sched) - 1
        for a in reversed(sorted(ctx.ckpts)):
            b = min(a + ctx.ckpt, nsteps)
            c0, o0, v0 = ctx.ckpts[a]
            c, o, v = c0.clone(), [t.clone() for t in o0], [t.clone() for t in v0]
            states = []
            for s in range(a, b):
                states.append((c.clone(), [t.clone() for t in o]))
                ck, dd = sched[s]
                plan.step_split(c, o, v, mass, cp, ck, dd)
            for s in reversed(range(a, b)):
                ck, dd = sched[s]
                plan.step_adjoint_split(*states[s - a], mass, cp, ck, dd, xb, vb)
        grad = torch.stack([xb[a].double() + ctx.vel_factor * vb[a].double() for a in range(3)])
        return grad, None, None, None, None, None, None, None, None, None, None


def loss_fn_split(psi, q, plan, ng, mass, c_poisson, dt, steps, target, vel_factor=1.0, ckpt=8):
    return PMLossSplit.apply(psi, q, plan, ng, mass, c_poisson, dt, steps, target, vel_factor, ckpt)
