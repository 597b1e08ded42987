"""torch.autograd.Function over the C-ABI adjoint window: test harness only.

The misfit J(T0) of an assimilation window and its gradient come from one
lbrb_adjoint_window call (forward + hand-written adjoint on the GPU); this
wrapper lets torch's own checking tools (gradcheck) drive them.
"""
import numpy as np
import torch


class WindowMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, T0, run, nsteps, K):
        J, grad = run.adjoint_window(T0.detach().cpu().numpy().astype(np.float64), nsteps, K)
        ctx.save_for_backward(torch.from_numpy(grad).to(T0))
        return T0.new_tensor(J)

    @staticmethod
    def backward(ctx, gJ):
        (grad,) = ctx.saved_tensors
        return gJ * grad, None, None, None
