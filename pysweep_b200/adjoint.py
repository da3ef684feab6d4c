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
import functools

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


class SweptHeatVar:
    """The same solve through the swept decomposition (the engine's prism,
    bridge and octahedron phases; Engine equations "heatvar",
    "heatvar_adjoint_mu" and "heatvar_adjoint", csrc/equations.cuh):

    * forward: u0 -> u_T with a courant number per cell, the state copied out
      every `every` steps (the checkpoints);
    * backward: for the segments from the last to the first, the segment's
      levels are recomputed from its checkpoint, storing each old level's
      Laplacian L(u_n) (ps_heatvar_recompute: the fused two-level forward
      kernels, faster than the swept forward where the fields fit in L2, and
      the same values); then an adjoint engine runs the segment backward
      through the swept decomposition.

    form="mu" (default): the adjoint in mu = C .* lambda,
    mu_n = mu_{n+1} + C .* L(mu_{n+1}), the forward step itself, so it runs in
    the forward's register-resident streams; the sum of mu_{n+1} .* L(u_n)
    accumulates in place, and lambda_0 = mu_0 ./ C, dJ/dC = sum ./ C at the
    end.  Same gradients as the standard kernels up to rounding (the products
    C .* lambda are formed in another place).
    form="lambda": lambda_n = lambda_{n+1} + L(C .* lambda_{n+1}),
    dJ/dC += lambda_{n+1} .* L(u_n) in the generic swept kernels; every cell
    sees the standard kernels' operations in the same order, so lambda_0 and
    dJ/dalpha equal theirs bitwise.

    The forward pass equals the standard forward bitwise in both forms.  The
    work runs on a stream of its own, ordered after the caller's current
    stream on entry and before it on return."""

    def __init__(self, nx, ny, every, blocksize=32, device=0, form="mu"):
        from .engine import Engine
        if form not in ("mu", "lambda"):
            raise ValueError(f"form {form!r}: 'mu' or 'lambda'")
        self.nx, self.ny, self.every, self.device, self.form = nx, ny, every, device, form
        # one stream for both engines (the recompute's Laplacians are read by
        # the adjoint engine's next run), ordered after the caller's stream
        self.stream = torch.cuda.Stream(device=device)
        self.fwd = Engine("heatvar", nx, ny, blocksize=blocksize, device=device)
        self.adj = Engine("heatvar_adjoint_mu" if form == "mu" else "heatvar_adjoint", nx, ny,
                          blocksize=blocksize, device=device)
        for e in (self.fwd, self.adj):
            e.set_stream(self.stream.cuda_stream)
        self.lap = None

    @staticmethod
    def levels_per_half_cycle(nx, ny, form="mu", device=0, blocksize=32):
        """The swept engines' levels per half-cycle (both engines use the
        same)."""
        return _levels_per_half_cycle(nx, ny, device, blocksize)

    def _enter(self):
        caller = torch.cuda.current_stream(self.device)
        self.stream.wait_stream(caller)
        return caller

    def _leave(self, caller, *outs):
        caller.wait_stream(self.stream)
        for t in outs:
            t.record_stream(caller)
        return outs

    def forward(self, u0, courant, nsteps, ck):
        """u_T; ck[k] receives the state after k*every steps."""
        caller = self._enter()
        with torch.cuda.stream(self.stream):
            f = self.fwd
            f.set_field(0, courant)
            f.set_field(1, None)
            f.set_state(u0)
            ck[0].copy_(u0)
            done, k = 0, 0
            while done < nsteps:
                n = min(self.every, nsteps - done)
                f.run(n)
                done += n
                k += 1
                if done < nsteps:
                    f.get_state(out=ck[k])
            out = torch.empty_like(u0)
            f.get_state(out=out)
        return self._leave(caller, out)[0]

    def backward(self, courant, ck, nsteps, lam_T):
        """(lambda_0, dJ/dC)."""
        nx, ny, every = self.nx, self.ny, self.every
        mu = self.form == "mu"
        caller = self._enter()
        with torch.cuda.stream(self.stream):
            if self.lap is None:
                self.lap = torch.empty((every, nx, ny), dtype=lam_T.dtype, device=lam_T.device)
                self.work = torch.empty((2, nx, ny), dtype=lam_T.dtype, device=lam_T.device)
            a = self.adj
            a.set_field(0, courant)
            a.set_field(1, self.lap)
            if mu:
                state = courant * lam_T                 # mu_T = C .* lambda_T
                acc = torch.zeros_like(lam_T)           # sum of mu_{n+1} .* L(u_n)
                a.set_field(2, acc)
            else:
                state = torch.zeros((2, nx, ny), dtype=lam_T.dtype, device=lam_T.device)
                state[0].copy_(lam_T)
            nseg = max(1, -(-nsteps // every))
            for sidx in range(nseg - 1, -1, -1):
                n0 = sidx * every
                length = min(n0 + every, nsteps) - n0
                if length <= 0:
                    continue
                # L(u_{n0}) .. L(u_{n0+length-1}) from the checkpoint (the
                # fused forward kernels: at sizes whose fields stay in L2 they
                # outrun the swept forward, and the values are the same)
                _call(_lib.lib().ps_heatvar_recompute, _p(courant), _p(ck[sidx]), _p(self.lap),
                      length, nx, ny, _p(self.work))
                a.set_global("LEN", length)
                a.set_state(state)
                a.run(length)          # segment end -> n0
                a.get_state(out=state)
            if mu:
                a.set_field(2, None)
                lam0, gC = state / courant, acc / courant
            else:
                lam0, gC = state[0].clone(), state[1].clone()
            # the Laplacian slab (every fields) goes back to torch's cache of
            # this stream; a cached solver does not hold it between solves
            a.set_field(1, None)
            self.lap = self.work = None
        return self._leave(caller, lam0, gC)

    def close(self):
        self.fwd.close()
        self.adj.close()


@functools.lru_cache(maxsize=None)
def _levels_per_half_cycle(nx, ny, device, blocksize):
    from .engine import Engine
    e = Engine("heatvar", nx, ny, blocksize=blocksize, device=device)
    h = e.tiling()["h"]
    e.close()
    return h


# Swept solvers of recent shapes, reused across solves: creating one
# allocates its engines' device buffers (synchronising the device), which
# costs as much as a short solve.  A solver evicted here lives on until no
# pending backward pass holds it.
_swept_cache = {}
_SWEPT_CACHE_MAX = 4


def _swept_solver(nx, ny, every, form, device):
    key = (nx, ny, every, form, device)
    sw = _swept_cache.pop(key, None)
    if sw is None:
        sw = SweptHeatVar(nx, ny, every, device=device, form=form)
    _swept_cache[key] = sw  # most recently used last
    while len(_swept_cache) > _SWEPT_CACHE_MAX:
        _swept_cache.pop(next(iter(_swept_cache)))
    return sw


def release_swept_solvers():
    """Drop the cached swept solvers; their device buffers are freed once no
    pending backward pass holds them."""
    _swept_cache.clear()


class HeatVarSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, alpha, nsteps, dt, dx, every, swept=False):
        u0 = u0.contiguous()
        alpha = alpha.contiguous()
        nx, ny = u0.shape
        if swept:
            courant = torch.empty_like(u0)
            _call(_lib.lib().ps_heatvar_courant, _p(alpha), _p(courant), nx, ny, dt, dx)
            form = "lambda" if swept == "lambda" else "mu"
            # checkpoint segments of whole half-cycles (the values do not
            # depend on the spacing; partial half-cycles cost a launch set
            # for few levels)
            h = SweptHeatVar.levels_per_half_cycle(nx, ny, form, u0.device.index or 0)
            every = max(h, every - every % h)
            sw = _swept_solver(nx, ny, every, form, u0.device.index or 0)
            ck = torch.empty((max(1, -(-nsteps // every)), nx, ny), dtype=u0.dtype,
                             device=u0.device)
            uT = sw.forward(u0, courant, nsteps, ck)
            ctx.sw = sw
        else:
            ck = torch.empty((max(1, -(-nsteps // every)), nx, ny), dtype=u0.dtype,
                             device=u0.device)
            courant = torch.empty_like(u0)
            work = torch.empty_like(u0)
            uT = torch.empty_like(u0)
            _call(_lib.lib().ps_heatvar_forward, _p(u0), _p(alpha), _p(uT), nx, ny, nsteps, dt,
                  dx, _p(courant), _p(work), _p(ck), every)
            ctx.sw = None
        ctx.save_for_backward(courant, ck)
        ctx.cfg = (nsteps, dt, dx, every, nx, ny)
        return uT

    @staticmethod
    def backward(ctx, grad_uT):
        courant, ck = ctx.saved_tensors
        nsteps, dt, dx, every, nx, ny = ctx.cfg
        g = grad_uT.contiguous()
        if ctx.sw is not None:
            lam0, gC = ctx.sw.backward(courant, ck, nsteps, g)
            ctx.sw = None
            # dJ/dalpha = dJ/dC * dt/dx/dx (scale_kernel's factor)
            return lam0, gC * (dt / dx / dx), None, None, None, None, None
        states = torch.empty((every, nx, ny), dtype=g.dtype, device=g.device)
        lamwork = torch.empty_like(g)
        lam0 = torch.empty_like(g)
        galpha = torch.empty_like(g)
        _call(_lib.lib().ps_heatvar_adjoint, _p(courant), _p(ck), every, _p(g), _p(lam0),
              _p(galpha), nx, ny, nsteps, dt, dx, _p(states), _p(lamwork))
        return lam0, galpha, None, None, None, None, None


def heat_solve(u0, alpha, nsteps, dt, dx, every=64, swept=False):
    """swept=False: the fused standard kernels (two levels per launch);
    swept=True or "mu": the swept decomposition with the adjoint in
    mu = C .* lambda (SweptHeatVar, register-resident streams); swept="lambda":
    the swept decomposition with the adjoint in lambda, bitwise equal to the
    standard kernels.  The forward values are bitwise equal in all three."""
    if swept not in (False, True, "mu", "lambda"):
        raise ValueError(f"swept={swept!r}: False, True, 'mu' or 'lambda'")
    return HeatVarSolve.apply(u0, alpha, int(nsteps), float(dt), float(dx), int(every),
                              swept if isinstance(swept, str) else bool(swept))


def heat_solve_reference(u0, alpha, nsteps, dt, dx):
    """The same update in plain torch (differentiable by autograd)."""
    c = alpha * dt / dx / dx
    u = u0
    for _ in range(nsteps):
        dxx = (torch.roll(u, -1, 0) - 2 * u) + torch.roll(u, 1, 0)
        dyy = (torch.roll(u, -1, 1) - 2 * u) + torch.roll(u, 1, 1)
        u = (c * dxx + c * dyy) + u
    return u
