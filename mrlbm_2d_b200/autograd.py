"""torch.autograd bridge to the adjoint of mean drag (mrlbm_adjoint_drag).

    J = mean_drag(sim, body_force, u_inlet, nsteps=8000, window=2000, checkpoint_every=100)
    J.backward()          # body_force.grad, u_inlet.grad from the hand-written adjoint kernels

`body_force` is a (2, nx, ny) tensor (x and y components per node), `u_inlet` a (ny,) tensor;
both may live on any device and be float32 or float64 (they are passed to the FP64 step as
float64).  The forward sets them on the simulation, runs the checkpointed forward and backward
passes once and keeps the gradients for `backward`; the simulation's state is not advanced.
"""
import numpy as np
import torch


class MeanDrag(torch.autograd.Function):
    @staticmethod
    def forward(ctx, body_force, u_inlet, sim, nsteps, window, checkpoint_every):
        sim.set_body_force(body_force.detach().to("cpu", torch.float64).numpy())
        sim.set_inlet_profile(u_inlet.detach().to("cpu", torch.float64).numpy())
        J, gb, gu = sim.adjoint_drag(nsteps, window, checkpoint_every, grads=True)
        ctx.save_for_backward(torch.from_numpy(gb).to(body_force.device, body_force.dtype),
                              torch.from_numpy(np.asarray(gu)).to(u_inlet.device, u_inlet.dtype))
        return torch.tensor(J, dtype=torch.float64, device=body_force.device)

    @staticmethod
    def backward(ctx, gJ):
        gb, gu = ctx.saved_tensors
        s = gJ.to(gb.dtype)
        return s * gb, s * gu, None, None, None, None


def mean_drag(sim, body_force, u_inlet, nsteps, window, checkpoint_every=100):
    """Differentiable mean drag over the last `window` of `nsteps` steps from the current state."""
    return MeanDrag.apply(body_force, u_inlet, sim, int(nsteps), int(window), int(checkpoint_every))
