"""The swept form of the differentiable variable-diffusivity heat solve
(adjoint.SweptHeatVar: the engine's heatvar, heatvar_adjoint_mu and
heatvar_adjoint equations through the prism / bridge / octahedron phases)
against the standard fused kernels (bitwise for the forward pass and the
lambda-form adjoint, to 1e-12 for the mu-form adjoint, which forms C * lambda
elsewhere) and against torch autograd."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fields(n, seed):
    import torch
    rng = np.random.default_rng(seed)
    x = np.arange(n) / n

    def fourier(modes=8):
        f = np.zeros((n, n))
        for _ in range(modes):
            k, l = rng.integers(1, 9, 2)
            f += rng.uniform(0, 1) * np.sin(2 * np.pi * (k * x[:, None] + l * x[None, :]) +
                                            rng.uniform(0, 2 * np.pi))
        return f / modes
    u0 = torch.tensor(fourier(), dtype=torch.float64, device="cuda")
    alpha = torch.tensor(1.0 + 0.5 * fourier(), dtype=torch.float64, device="cuda")
    target = torch.tensor(fourier(), dtype=torch.float64, device="cuda")
    return u0, alpha, target


def _grads(n, steps, every, swept, seed):
    import torch
    from pysweep_b200.adjoint import heat_solve
    u0, alpha, target = _fields(n, seed)
    dx = 1.0 / n
    dt = 0.2 * dx * dx / 1.5
    x = u0.clone().requires_grad_(True)
    y = alpha.clone().requires_grad_(True)
    uT = heat_solve(x, y, steps, dt, dx, every, swept=swept)
    loss = 0.5 * ((uT - target) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return uT.detach(), x.grad, y.grad


CASES = [(256, 100, 32), (256, 57, 16), (128, 40, 64), (512, 30, 7)]


@pytest.mark.parametrize("n,steps,every", CASES)
def test_swept_lambda_form_equals_standard_bitwise(n, steps, every):
    a = _grads(n, steps, every, False, n + steps)
    b = _grads(n, steps, every, "lambda", n + steps)
    for name, x, y in zip(("u_T", "dJ/du0", "dJ/dalpha"), a, b):
        assert bool((x == y).all()), (name, (x - y).abs().max().item(), y.abs().max().item())


@pytest.mark.parametrize("n,steps,every", CASES)
def test_swept_mu_form_matches_standard(n, steps, every):
    a = _grads(n, steps, every, False, n + steps)
    b = _grads(n, steps, every, "mu", n + steps)
    assert bool((a[0] == b[0]).all())  # the forward pass: bitwise
    for name, x, y in zip(("dJ/du0", "dJ/dalpha"), a[1:], b[1:]):
        rel = ((x - y).abs().max() / x.abs().max()).item()
        assert rel < 1e-12, (name, rel)


def test_swept_gradients_match_torch_autograd():
    import torch
    from pysweep_b200.adjoint import heat_solve, heat_solve_reference
    n, steps = 128, 60
    u0, alpha, target = _fields(n, 5)
    dx = 1.0 / n
    dt = 0.2 * dx * dx / 1.5
    g = []
    for f in (lambda a, b: heat_solve(a, b, steps, dt, dx, 16, swept="mu"),
              lambda a, b: heat_solve_reference(a, b, steps, dt, dx)):
        x = u0.clone().requires_grad_(True)
        y = alpha.clone().requires_grad_(True)
        loss = 0.5 * ((f(x, y) - target) ** 2).sum()
        loss.backward()
        g.append((x.grad, y.grad))
    for mine, ref in zip(g[0], g[1]):
        rel = ((mine - ref).abs().max() / ref.abs().max()).item()
        assert rel < 1e-11, rel


def test_heatvar_engines_swept_equal_standard():
    """The two equations through the engine: swept == standard, bitwise, for
    every stored frame (heatvar) and for lambda and dJ/dC (the adjoint)."""
    import torch
    from pysweep_b200 import Engine
    n, nl = 192, 29
    u0, alpha, _ = _fields(n, 9)
    C = (alpha * 1e-1).contiguous()
    lap = {m: torch.zeros((nl, n, n), dtype=torch.float64, device="cuda") for m in ("swept", "standard")}
    fr = {}
    for mode in ("swept", "standard"):
        e = Engine("heatvar", n, n, blocksize=32)
        e.set_field(0, C)
        e.set_field(1, lap[mode])
        e.set_global("LEN", nl)
        e.set_state(u0)
        fr[mode] = np.zeros((nl, 1, n, n))
        e.run(nl, mode=mode, frames=fr[mode])
        e.close()
    assert np.array_equal(fr["swept"], fr["standard"])
    assert bool((lap["swept"] == lap["standard"]).all())
    st = torch.stack([u0, torch.zeros_like(u0)]).contiguous()
    out = {}
    for mode in ("swept", "standard"):
        a = Engine("heatvar_adjoint", n, n, blocksize=32)
        a.set_field(0, C)
        a.set_field(1, lap[mode])
        a.set_global("LEN", nl)
        a.set_state(st)
        a.run(nl, mode=mode)
        out[mode] = a.get_state()
        a.close()
    assert np.array_equal(out["swept"], out["standard"])
    assert np.abs(out["swept"][1]).max() > 0


@pytest.mark.parametrize("bs,n", [(32, 256), (16, 192)])
def test_register_streams_per_cell_courant(bs, n):
    """heatvar and heatvar_adjoint_mu in the register-resident streams against
    the generic swept kernels (threads=256) and the standard path, bitwise:
    the fields, every recomputed Laplacian and the adjoint's sum."""
    import torch
    from pysweep_b200 import Engine
    nl = 40
    u0, alpha, _ = _fields(n, 11 + bs)
    C = (alpha * 1e-1).contiguous()
    res = {}
    for key, mode, threads in (("fast", "swept", 0), ("generic", "swept", 256),
                               ("standard", "standard", 0)):
        lap = torch.zeros((nl, n, n), dtype=torch.float64, device="cuda")
        e = Engine("heatvar", n, n, blocksize=bs)
        if threads:
            e.configure(threads=threads)
        e.set_field(0, C)
        e.set_field(1, lap)
        e.set_global("LEN", nl)
        e.set_state(u0)
        e.run(nl, mode=mode)
        u = e.get_state()
        e.close()
        acc = torch.zeros_like(u0)
        a = Engine("heatvar_adjoint_mu", n, n, blocksize=bs)
        if threads:
            a.configure(threads=threads)
        a.set_field(0, C)
        a.set_field(1, lap)
        a.set_field(2, acc)
        a.set_global("LEN", nl)
        a.set_state(u0)
        a.run(nl, mode=mode)
        mu = a.get_state()
        a.close()
        torch.cuda.synchronize()
        res[key] = (u, lap.cpu().numpy(), mu, acc.cpu().numpy())
    for key in ("generic", "standard"):
        for x, y in zip(res["fast"], res[key]):
            assert np.array_equal(x, y), key
    assert np.abs(res["fast"][3]).max() > 0


def test_heatvar_needs_its_fields_and_levels():
    import torch
    from pysweep_b200 import Engine
    from pysweep_b200._lib import PySweepError
    e = Engine("heatvar_adjoint", 64, 64, blocksize=16)
    e.set_state(np.zeros((2, 64, 64)))
    with pytest.raises(PySweepError):
        e.run(4)  # no fields
    C = torch.full((64, 64), 0.1, dtype=torch.float64, device="cuda")
    lap = torch.zeros((4, 64, 64), dtype=torch.float64, device="cuda")
    e.set_field(0, C)
    e.set_field(1, lap)
    e.set_global("LEN", 4)
    with pytest.raises(PySweepError):
        e.run(5)  # more levels than the Laplacians hold
    e.run(4)
    e.synchronize()
    e.close()


@pytest.mark.parametrize("length", [1, 6, 13])
def test_fused_recompute_laplacians_equal_swept_engine(length):
    """ps_heatvar_recompute (the fused forward kernels) stores the same
    Laplacians as the swept heatvar engine, bitwise."""
    import ctypes

    import torch
    from pysweep_b200 import Engine, _lib
    n = 256
    u0, alpha, _ = _fields(n, 21 + length)
    C = (alpha * 1e-1).contiguous()
    lap_swept = torch.zeros((length, n, n), dtype=torch.float64, device="cuda")
    e = Engine("heatvar", n, n, blocksize=32)
    e.set_field(0, C)
    e.set_field(1, lap_swept)
    e.set_global("LEN", length)
    e.set_state(u0)
    e.run(length)
    e.synchronize()
    e.close()
    lap_fused = torch.zeros_like(lap_swept)
    work = torch.empty((2, n, n), dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = _lib.lib().ps_heatvar_recompute(p(C), p(u0), p(lap_fused), length, n, n, p(work),
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                         err, 256)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    assert bool((lap_fused == lap_swept).all())


def test_cached_swept_solver_serves_interleaved_solves():
    """Two swept solves of one shape share a cached solver: both forward
    passes first, then the backward passes in reverse order, give each solve
    the gradients it gets alone."""
    import torch
    from pysweep_b200.adjoint import heat_solve, release_swept_solvers
    n, steps, every = 256, 50, 24
    dx = 1.0 / n
    dt = 0.2 * dx * dx / 1.5
    alone = [_grads(n, steps, every, "mu", seed) for seed in (3, 4)]
    runs = []
    for seed in (3, 4):
        u0, alpha, target = _fields(n, seed)
        x = u0.clone().requires_grad_(True)
        y = alpha.clone().requires_grad_(True)
        loss = 0.5 * ((heat_solve(x, y, steps, dt, dx, every, swept="mu") - target) ** 2).sum()
        runs.append((loss, x, y))
    for loss, _, _ in reversed(runs):
        loss.backward()
    torch.cuda.synchronize()
    for (loss, x, y), (_, gx, gy) in zip(runs, alone):
        assert bool((x.grad == gx).all()) and bool((y.grad == gy).all())
    release_swept_solvers()
