"""torch.autograd.Function over the discrete adjoint (fv_adjoint_*), used
only for gradient checks (torch.autograd.gradcheck): forward runs the
FP64_EXACT time loop and returns the loss, backward scales the adjoint
gradient computed in the same call."""
import torch

import fvgpu


class InflowLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, adjoint: "fvgpu.Adjoint"):
        t = theta.detach().cpu().double().numpy()
        if theta.requires_grad:
            loss, grad = adjoint.gradient(t)
            ctx.save_for_backward(torch.from_numpy(grad).to(theta))
        else:
            loss = adjoint.loss(t)
        return theta.new_tensor(loss)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad_out * grad, None


def inflow_loss(theta: torch.Tensor, adjoint: "fvgpu.Adjoint") -> torch.Tensor:
    return InflowLoss.apply(theta, adjoint)
