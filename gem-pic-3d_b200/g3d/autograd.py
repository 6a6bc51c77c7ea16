"""A thin torch.autograd.Function over the adjoint march (g3d_adjoint), for gradient checks with torch's tools.

J = sum w p_z / sum w over the live beam after K s-steps, as a function of the laser mode coefficients a (every
grid laser's spectrum added at init is multiplied per stored mode by a) and of offsets added to the bunch's
momenta. Each call runs, on a fresh context of the current CUDA device, the forward with per-level checkpoints
and the reverse sweep; backward hands out the stored gradients times the incoming one. torch carries the
tensors only: the forward and the adjoint are the library's.

Inputs: coef, float64 [ny, nx/2 + 1, 2] (the real and imaginary parts of a); dp, float64 [np, 3] (added to the
momenta as loaded when through_start, the derivative then running through the start field the bunch makes at
init; else added right after init, the start field held). The output is J - j0 for a constant j0: with j0 near
J the subtraction is exact per particle and the difference keeps the digits a central difference needs
(J ~ gamma would round each evaluation to 1e-16 gamma).
"""
import math

import numpy as np
import torch

from .sim import Simulation


def _evaluate(coef, dp, cfg, precision, exact, through_start):
    sim = Simulation(cfg, precision=precision)
    try:
        sim.load_bunch()
        p = sim.host_particles()
        if dp.shape != (len(p), 3):
            raise ValueError(f"dp must be [{len(p)}, 3], not {list(dp.shape)}")

        def offset():
            q = sim.host_particles()
            q["px"] += dp[:, 0]; q["py"] += dp[:, 1]; q["pz"] += dp[:, 2]
            sim.set_particles(q)
        if through_start:
            offset()
        sim.set_laser_modes(coef[..., 0] + 1j * coef[..., 1])
        if exact:
            sim.set_exact_fields(True)
        sim.init_fields()
        if not through_start:
            offset()
        _, gm, gp = sim.adjoint(cfg.steps, through_start=through_start)
        return sim.host_particles(), gm, gp
    finally:
        sim.close()


class MarchObjective(torch.autograd.Function):
    """MarchObjective.apply(coef, dp, cfg, precision="fp64", exact=True, through_start=True, j0=0.0) -> J - j0."""

    @staticmethod
    def forward(ctx, coef, dp, cfg, precision="fp64", exact=True, through_start=True, j0=0.0):
        c = coef.detach().to("cpu", torch.float64).numpy()
        d = dp.detach().to("cpu", torch.float64).numpy()
        if c.shape != (cfg.ny, cfg.nx // 2 + 1, 2):
            raise ValueError(f"coef must be [{cfg.ny}, {cfg.nx // 2 + 1}, 2], not {list(c.shape)}")
        q, gm, gp = _evaluate(c, d, cfg, precision, exact, through_start)
        a = q["alive"] == 1
        w, pz = q["w"][a], q["pz"][a]
        val = math.fsum(w * (pz - j0)) / math.fsum(w)
        ctx.save_for_backward(torch.from_numpy(np.stack([gm.real, gm.imag], axis=-1)).to(coef.device),
                              torch.from_numpy(gp).to(dp.device))
        return torch.tensor(val, dtype=torch.float64, device=coef.device)

    @staticmethod
    def backward(ctx, g):
        gm, gp = ctx.saved_tensors
        return g * gm, g * gp, None, None, None, None, None
