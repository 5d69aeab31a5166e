"""torch.autograd binding of the engine's discrete adjoint.

``seismograms(lam, mu, rho, model, nsteps)`` runs the FP64 engine forward with
device checkpoints and returns the station seismograms as a tensor; its
backward runs ``axg_adjoint_run`` (time-reversed adjoint with per-segment
recomputation) and returns dJ/d(lambda), dJ/d(mu) per element point and
dJ/d(rho) per element point (through the point masses, M_p = sum rho_eq ifact_eq,
Material::getMass). Tensors live on the CPU; the engine does the work on the GPU.
"""
import copy

import numpy as np
import torch

from .solver import Solver


class _Seismograms(torch.autograd.Function):
    @staticmethod
    def forward(ctx, lam, mu, rho, model, nsteps, interval):
        m = copy.copy(model)
        ne = model.n_solid_elements
        m.se_moduli = np.stack([lam.detach().cpu().numpy(), mu.detach().cpu().numpy()], axis=1).reshape(-1)
        m.se_mat_off = np.arange(ne, dtype=np.int64) * 50
        ifact = model.se_geom[:, 5, :]
        r = rho.detach().cpu().numpy()
        mass = np.zeros(len(model.sp_nr))
        np.add.at(mass, model.se_pts.ravel(), (r * ifact).ravel())
        m.sp_mass = mass
        s = Solver(m, "fp64")
        s.forward_checkpointed(int(nsteps), int(interval))
        seis = s.seismograms()
        ctx.solver = s
        ctx.model = model
        return torch.from_numpy(seis)

    @staticmethod
    def backward(ctx, gseis):
        s = ctx.solver
        g = s.adjoint(gseis.detach().cpu().numpy().astype(np.float64))
        s.close()
        model = ctx.model
        gl = torch.from_numpy(g["moduli"][:, 0, :].copy())
        gm = torch.from_numpy(g["moduli"][:, 1, :].copy())
        grho = torch.from_numpy(g["mass"][model.se_pts] * model.se_geom[:, 5, :])
        return gl, gm, grho, None, None, None


def seismograms(lam, mu, rho, model, nsteps, interval=100):
    """Differentiable seismograms (nrecords, nstations, 3) of an isotropic 1-D model."""
    return _Seismograms.apply(lam, mu, rho, model, nsteps, interval)
