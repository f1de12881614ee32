"""torch.autograd binding of the CGFDM adjoint (cgfdm_gradient, via ctypes).

    J = misfit(vp, vs, rho, session, observed)
    J.backward()          # vp.grad, vs.grad, rho.grad

vp, vs, rho are the medium on the interior grid, [nz][ny][nx] tensors (any
device; float32 on the host at the boundary), observed the data the run's
stations should record, [n_stations][NT][3].  J = 1/2 sum (v - d)^2 over the
recorded station velocities.  The medium is handed to the session with
cgfdm_set_medium (the 3-cell halo filled from the nearest interior point,
where the stencil never reads it), and, when any input needs a gradient,
cgfdm_gradient runs the forward and the adjoint at once; backward only
scales the stored gradient.  The gradient is zero inside the PML layers.
"""

from __future__ import annotations

import numpy as np
import torch

from . import Session


def _padded_medium(vp: np.ndarray, vs: np.ndarray, rho: np.ndarray) -> np.ndarray:
    med = np.stack([vs, vp, rho], axis=-1).astype(np.float32)
    return np.pad(med, ((3, 3), (3, 3), (3, 3), (0, 0)), mode="edge")


class SeismogramMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vp, vs, rho, session: Session, observed, checkpoint_every: int = 100):
        host = [t.detach().to("cpu", torch.float32).numpy() for t in (vp, vs, rho)]
        session.set_medium(_padded_medium(*host))
        obs = observed.detach().to("cpu", torch.float32).numpy() if torch.is_tensor(observed) else observed
        if any(ctx.needs_input_grad[:3]):
            J, g = session.gradient(obs, checkpoint_every)
            ctx.grads = [torch.from_numpy(g[c]).to(t.device, t.dtype) for c, t in enumerate((vp, vs, rho))]
        else:
            session.run(session.info.NT)
            v = session.stations()[:, :, :3].astype(np.float64)
            J = 0.5 * float(np.sum((v - np.asarray(obs, np.float64)) ** 2))
            ctx.grads = [None, None, None]
        return torch.tensor(J, dtype=torch.float64, device=vp.device)

    @staticmethod
    def backward(ctx, gJ):
        out = [None if g is None else g * gJ.to(g.dtype) for g in ctx.grads]
        return out[0], out[1], out[2], None, None, None


def misfit(vp, vs, rho, session: Session, observed, checkpoint_every: int = 100):
    """J(vp, vs, rho) as a differentiable torch scalar (float64)."""
    return SeismogramMisfit.apply(vp, vs, rho, session, observed, checkpoint_every)
