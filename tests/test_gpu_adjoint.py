"""The hand-written adjoint of the variable-diffusivity heat solve against
torch autograd through the plain stencil and against central finite
differences."""
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
            f += rng.uniform(0, 1) * np.sin(2 * np.pi * (k * x[:, None] + l * x[None, :]) + rng.uniform(0, 2 * np.pi))
        return f / modes
    u0 = torch.tensor(fourier(), dtype=torch.float64, device="cuda")
    alpha = torch.tensor(1.0 + 0.5 * fourier(), dtype=torch.float64, device="cuda")
    target = torch.tensor(fourier(), dtype=torch.float64, device="cuda")
    return u0, alpha, target


def test_forward_matches_plain_stencil_bitwise():
    from pysweep_b200.adjoint import heat_solve, heat_solve_reference
    n, steps = 256, 57
    u0, alpha, _ = _fields(n, 1)
    dx = 1.0 / n
    dt = 0.2 * dx * dx / 1.5
    a = heat_solve(u0, alpha, steps, dt, dx, every=16)
    b = heat_solve_reference(u0, alpha, steps, dt, dx)
    assert bool((a == b).all())


@pytest.mark.parametrize("every", [16, 64, 7])
def test_gradients_match_torch_autograd(every):
    import torch
    from pysweep_b200.adjoint import heat_solve, heat_solve_reference
    n, steps = 256, 100
    u0, alpha, target = _fields(n, 2)
    dx = 1.0 / n
    dt = 0.2 * dx * dx / 1.5
    g = []
    for f in (lambda a, b: heat_solve(a, b, steps, dt, dx, every), lambda a, b: heat_solve_reference(a, b, steps, dt, dx)):
        x = u0.clone().requires_grad_(True)
        y = alpha.clone().requires_grad_(True)
        loss = 0.5 * ((f(x, y) - target) ** 2).sum()
        loss.backward()
        g.append((x.grad, y.grad))
    for mine, ref in zip(g[0], g[1]):
        rel = ((mine - ref).abs().max() / ref.abs().max()).item()
        assert rel < 1e-11, rel


def test_fused_and_single_step_backward_agree_bitwise():
    """Segments of one step run only the one-step kernels; longer segments run
    the two-step fused recompute and adjoint kernels (plus one single step for
    odd lengths).  Both evaluate every cell with the same operations."""
    from pysweep_b200.adjoint import heat_solve
    n, steps = 128, 37
    u0, alpha, target = _fields(n, 4)
    dx = 1.0 / n
    dt = 0.2 * dx * dx / 1.5
    grads = []
    for every in (1, 64, 9):
        x = u0.clone().requires_grad_(True)
        y = alpha.clone().requires_grad_(True)
        (0.5 * ((heat_solve(x, y, steps, dt, dx, every) - target) ** 2).sum()).backward()
        grads.append((x.grad, y.grad))
    for g in grads[1:]:
        assert bool((g[0] == grads[0][0]).all()) and bool((g[1] == grads[0][1]).all())


def test_gradients_match_central_differences():
    """Directional derivatives against Richardson-extrapolated central
    differences, (4 D(h/2) - D(h)) / 3 with D(h) = (J(+h) - J(-h)) / 2h, along
    unit-norm directions.  The truncation error is O(h^4) (J is exactly
    quadratic in u0, and smooth in alpha); the roundoff of the four J values
    (J is a few hundred here) is about 1.5 * eps * J / h.  The test allows
    1e-7 relative plus 20 * eps * J / h."""
    import torch
    from pysweep_b200.adjoint import heat_solve
    n, steps, h = 256, 200, 1e-2
    u0, alpha, target = _fields(n, 3)
    dx = 1.0 / n
    dt = 0.2 * dx * dx / 1.5

    def J(a, b):
        return 0.5 * ((heat_solve(a, b, steps, dt, dx, 64) - target) ** 2).sum().item()

    def richardson(f):
        d = lambda e: (f(e) - f(-e)) / (2 * e)  # noqa: E731
        return (4 * d(h / 2) - d(h)) / 3

    x = u0.clone().requires_grad_(True)
    y = alpha.clone().requires_grad_(True)
    (0.5 * ((heat_solve(x, y, steps, dt, dx, 64) - target) ** 2).sum()).backward()
    gen = torch.Generator(device="cuda").manual_seed(0)
    for _ in range(4):
        du = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=gen)
        da = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=gen)
        du /= du.norm()
        da /= da.norm()
        fd_u = richardson(lambda e: J(u0 + e * du, alpha))
        fd_a = richardson(lambda e: J(u0, alpha + e * da))
        an_u = (x.grad * du).sum().item()
        an_a = (y.grad * da).sum().item()
        round_off = 20 * np.finfo(np.float64).eps * J(u0, alpha) / h
        assert abs(fd_u - an_u) <= 1e-7 * abs(an_u) + round_off, (fd_u, an_u)
        assert abs(fd_a - an_a) <= 1e-7 * abs(an_a) + round_off, (fd_a, an_a)
