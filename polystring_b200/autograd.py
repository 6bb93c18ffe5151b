"""torch.autograd harness over the C ABI adjoint: (wA, wB) -> (phiA, phiB, Q)
of Model_AB's forward map (src/Model_AB.cc:186-199 at fixed fields), with
backward = ps_model_ab_grad_w.

    phiA, phiB, Q = DensityMap.apply(wA, wB, model)     # float64 CPU tensors
    loss = ((phiA - phi_target) ** 2).sum()
    loss.backward()                                      # wA.grad, wB.grad
"""
import numpy as np
import torch


class DensityMap(torch.autograd.Function):
    @staticmethod
    def forward(ctx, wA, wB, model):
        fA = wA.detach().cpu().numpy().copy()
        fB = wB.detach().cpu().numpy().copy()
        model.set_fields(fA, fB)
        model.forward()
        ctx.model = model
        ctx.fields = (fA, fB)
        phiA = torch.from_numpy(model.get("phiA"))
        phiB = torch.from_numpy(model.get("phiB"))
        Q = torch.tensor(model.Q(), dtype=torch.float64)
        return phiA, phiB, Q

    @staticmethod
    def backward(ctx, gphiA, gphiB, gQ):
        m = ctx.model
        m.set_fields(*ctx.fields)       # the model may have moved on since forward()
        gA, gB = m.grad_w(np.ascontiguousarray(gphiA.detach().cpu().numpy()),
                          np.ascontiguousarray(gphiB.detach().cpu().numpy()), float(gQ))
        return torch.from_numpy(gA), torch.from_numpy(gB), None
