"""A thin torch.autograd binding of tmfqs_gpu_adjoint_gradient, used to check
the adjoint gradient through torch's own machinery (not a compute path: the
forward and backward both run inside the C ABI call).

    E = CircuitExpectation.apply(thetas, make_state, make_ops, masks, weights)
    E.backward()          # thetas.grad = dE/dthetas from the adjoint sweep

`make_state()` returns a GpuState holding the input state; `make_ops(values)`
returns the op list whose i-th CPHASE op carries values[i].
"""
import numpy as np
import torch


class CircuitExpectation(torch.autograd.Function):
    @staticmethod
    def forward(ctx, thetas, make_state, make_ops, masks, weights, checkpoint_every=0):
        ops = make_ops(thetas.detach().cpu().numpy().astype(np.float64))
        g = make_state()
        try:
            e, grads = g.adjoint_gradient(ops, masks, weights, checkpoint_every)
        finally:
            g.close()
        ctx.save_for_backward(torch.as_tensor(grads, dtype=thetas.dtype, device=thetas.device))
        return thetas.new_tensor(e)

    @staticmethod
    def backward(ctx, grad_e):
        (grads,) = ctx.saved_tensors
        return grad_e * grads, None, None, None, None, None
