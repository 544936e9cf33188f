"""torch.autograd wrapper of the library's reverse sweep (test harness only).

ProbeLoss(f1, uvel) = sum over probes of |u - u_target|^2 after the run of a
lbm_b200.adjoint.ProbeProblem; its backward is the library's checkpointed
adjoint sweep (no torch autograd graph through the kernels)."""
import torch


class ProbeLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f1, uvel, f2, problem, target):
        u = problem.forward(f1, f2, uvel)
        ctx.problem = problem
        ctx.save_for_backward(u, target)
        return ((u.double() - target.double()) ** 2).sum()

    @staticmethod
    def backward(ctx, g):
        u, target = ctx.saved_tensors
        fg, ug = ctx.problem.backward((2.0 * (u.double() - target.double()) * g).float())
        return fg, ug, None, None, None


def probe_loss(f1, uvel, f2, problem, target):
    return ProbeLoss.apply(f1, uvel, f2, problem, target)
