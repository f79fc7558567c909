"""torch.autograd bindings of the energy and force-matching gradients.

A thin layer for fitting harnesses: the forward pass sets the metal
parameters (and optionally the positions) of a Simulation, runs one force
evaluation on the GPU through the C ABI, and the backward pass returns the
adjoint gradients of capac_energy_grad / capac_force_match_grad.  Tensors
are FP64 on the CPU; the simulation state lives on the GPU.  No torch
operation runs on the hot path.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from . import PARAMS, Simulation


def _apply(sim: Simulation, params: torch.Tensor, positions: Optional[torch.Tensor]) -> None:
    """Set the parameters (PARAMS order; a width of 0 follows its C or alpha)."""
    p = params.detach().cpu().double().numpy()
    if p.shape != (len(PARAMS),):
        raise ValueError(f"params must have shape ({len(PARAMS)},) in the order {PARAMS}")
    for name, v in zip(PARAMS, p):
        v = float(v)
        if name in ("cpim_rq", "cpim_rp") and v == 0.0:
            if sim.param_get(name + "_tied") == 0.0:
                sim.param_set(name, 0.0)
        elif sim.param_get(name) != v:
            sim.param_set(name, v)
    if positions is not None:
        r = positions.detach().cpu().double().numpy()
        for a, k in enumerate(("rx", "ry", "rz")):
            sim.set(k, np.ascontiguousarray(r[:, a]))
    if sim.desc.n_mat > 0:  # a solve from zero: the reference's warm-start early exit stays out
        sim.set("vec_pq", np.zeros(sim.desc.n_mat))
    sim.force()


def _grad_vector(g: dict, params: torch.Tensor) -> torch.Tensor:
    """The parameter gradient in PARAMS order; a tied width (entry 0) gets 0,
    its share being inside the gradient of C or alpha."""
    out = torch.tensor([g[n] for n in PARAMS], dtype=torch.float64)
    for n in ("cpim_rq", "cpim_rp"):
        k = PARAMS.index(n)
        if float(params[k]) == 0.0:
            out[k] = 0.0
    return out


def current_params(sim: Simulation, tied_widths: bool = True) -> torch.Tensor:
    """The simulation's metal parameters as a tensor in PARAMS order; with
    tied_widths the width entries are 0 (they follow C and alpha, whose
    gradients then include the widths' share)."""
    vals = [sim.param_get(n) for n in PARAMS]
    if tied_widths:
        vals[PARAMS.index("cpim_rq")] = vals[PARAMS.index("cpim_rp")] = 0.0
    return torch.tensor(vals, dtype=torch.float64)


class Energy(torch.autograd.Function):
    """E(params, positions): the sum of the energy terms potential[1..14]."""

    @staticmethod
    def forward(ctx, params, positions, sim):
        _apply(sim, params, positions)
        e = float(sim.get("potential")[1:].sum())
        g, gr = sim.energy_grad(positions=positions is not None)
        ctx.save_for_backward(_grad_vector(g, params.detach()),
                              torch.from_numpy(gr) if gr is not None else torch.zeros(0))
        ctx.has_pos = positions is not None
        return torch.tensor(e, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        gp, gr = ctx.saved_tensors
        return grad_out * gp, (grad_out * gr if ctx.has_pos else None), None


class ForceMatchLoss(torch.autograd.Function):
    """mean((F(params, positions) - target)^2) over atoms and axes."""

    @staticmethod
    def forward(ctx, params, positions, target, sim):
        _apply(sim, params, positions)
        t = target.detach().cpu().double().numpy()
        want_pos = positions is not None
        out = sim.force_match_grad(t, positions=want_pos)
        loss, g = out[0], out[1]
        f = torch.from_numpy(sim.forces())
        ctx.save_for_backward(_grad_vector(g, params.detach()),
                              torch.from_numpy(out[2]) if want_pos else torch.zeros(0), f, target.detach().double())
        ctx.has_pos = want_pos
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        gp, gr, f, t = ctx.saved_tensors
        g_target = -2.0 * (f - t) / f.numel()
        return grad_out * gp, (grad_out * gr if ctx.has_pos else None), grad_out * g_target, None


def energy(sim: Simulation, params: torch.Tensor, positions: Optional[torch.Tensor] = None) -> torch.Tensor:
    return Energy.apply(params, positions, sim)


def force_match_loss(sim: Simulation, params: torch.Tensor, target: torch.Tensor,
                     positions: Optional[torch.Tensor] = None) -> torch.Tensor:
    return ForceMatchLoss.apply(params, positions, target, sim)
