"""A thin torch.autograd.Function over the hand-written adjoint (ctc_grad,
FP64): the masked CP loss 1/2 ||P_Omega(X - [[U_1, ..., U_d]])||^2 +
lambda sum ||U_m||^2 of a fixed sparse tensor as a function of the factor
matrices, whose backward pass is the adjoint kernel's gradient.  It exists
so that torch.autograd.gradcheck (central finite differences in FP64) can
check the kernel; training uses ctc_fo / FirstOrder directly."""
from __future__ import annotations

import torch

from . import api


class MaskedCPLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, tensor, context, lam, *factors):
        dims = [int(f.shape[0]) for f in factors]
        rank = int(factors[0].shape[1])
        model = api.Model(dims, rank)
        for m, f in enumerate(factors):
            model.set(m, f.detach().cpu().double().numpy())
        grads, obj = api.grad(context, tensor, model, lam)
        model.free()
        ctx.save_for_backward(*[torch.from_numpy(g).to(dtype=f.dtype, device=f.device)
                                for g, f in zip(grads, factors)])
        return torch.tensor(obj, dtype=factors[0].dtype, device=factors[0].device)

    @staticmethod
    def backward(ctx, gout):
        return (None, None, None) + tuple(gout * g for g in ctx.saved_tensors)


def masked_cp_loss(tensor: api.Tensor, context: api.Context, lam: float, *factors):
    return MaskedCPLoss.apply(tensor, context, lam, *factors)
