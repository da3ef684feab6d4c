"""Differentiable heat solve with a spatially varying diffusivity.

``heat_solve(u0, alpha, nsteps, dt, dx, every=64)`` returns u after `nsteps`
forward-Euler steps of u_t = alpha(x,y) * (u_xx + u_yy) on the
periodic grid (per-cell update in the heat plugin's operation order with
courant = alpha*dt/dx/dx).  It is a ``torch.autograd.Function``: the backward
pass runs the hand-written adjoint kernels (ps_heatvar_adjoint), recomputing
each `every`-step segment from the checkpoints the forward pass stored, and
returns gradients with respect to u0 and alpha.  Tensors are FP64 CUDA
tensors of shape (nx, ny), ny a multiple of 64.
"""
import ctypes

import torch

from . import _lib


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _call(fn, *args):
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(*args, ctypes.c_void_p(stream), err, 256)
    if rc != 0:
        raise _lib.PySweepError(rc, err.value.decode())


class HeatVarSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, alpha, nsteps, dt, dx, every):
        u0 = u0.contiguous()
        alpha = alpha.contiguous()
        nx, ny = u0.shape
        nseg = max(1, -(-nsteps // every))
        courant = torch.empty_like(u0)
        work = torch.empty_like(u0)
        ck = torch.empty((nseg, nx, ny), dtype=u0.dtype, device=u0.device)
        uT = torch.empty_like(u0)
        _call(_lib.lib().ps_heatvar_forward, _p(u0), _p(alpha), _p(uT), nx, ny, nsteps, dt, dx,
              _p(courant), _p(work), _p(ck), every)
        ctx.save_for_backward(courant, ck)
        ctx.cfg = (nsteps, dt, dx, every, nx, ny)
        return uT

    @staticmethod
    def backward(ctx, grad_uT):
        courant, ck = ctx.saved_tensors
        nsteps, dt, dx, every, nx, ny = ctx.cfg
        g = grad_uT.contiguous()
        states = torch.empty((every, nx, ny), dtype=g.dtype, device=g.device)
        lamwork = torch.empty_like(g)
        lam0 = torch.empty_like(g)
        galpha = torch.empty_like(g)
        _call(_lib.lib().ps_heatvar_adjoint, _p(courant), _p(ck), every, _p(g), _p(lam0),
              _p(galpha), nx, ny, nsteps, dt, dx, _p(states), _p(lamwork))
        return lam0, galpha, None, None, None, None


def heat_solve(u0, alpha, nsteps, dt, dx, every=64):
    return HeatVarSolve.apply(u0, alpha, int(nsteps), float(dt), float(dx), int(every))


def heat_solve_reference(u0, alpha, nsteps, dt, dx):
    """The same update in plain torch (differentiable by autograd)."""
    c = alpha * dt / dx / dx
    u = u0
    for _ in range(nsteps):
        dxx = (torch.roll(u, -1, 0) - 2 * u) + torch.roll(u, 1, 0)
        dyy = (torch.roll(u, -1, 1) - 2 * u) + torch.roll(u, 1, 1)
        u = (c * dxx + c * dyy) + u
    return u
