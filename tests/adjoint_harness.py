"""Check harness for the device adjoint: the head observable as a
torch.autograd.Function of relative parameter changes x, p = p0 (1 + x).
forward runs the program on the device (a5a_forward); backward returns the
device adjoint's gradient (a5a_gradient). Only the checks use it."""
import numpy as np
import torch


class HeadZ(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, adj, p0):
        p = p0 * (1.0 + x.detach().cpu().numpy())
        if ctx.needs_input_grad[0]:
            J, g = adj.gradient(p)
        else:
            J, g = adj.value(p), np.zeros(len(p0))
        ctx.save_for_backward(torch.from_numpy(np.asarray(g * p0)))
        return x.new_tensor(J)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g.to(grad_out.dtype), None, None


def head_z(x: torch.Tensor, adj, p0: np.ndarray) -> torch.Tensor:
    return HeadZ.apply(x, adj, p0)
