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


def test_gradients_match_central_differences():
    import torch
    from pysweep_b200.adjoint import heat_solve
    n, steps, h = 256, 200, 1e-6
    u0, alpha, target = _fields(n, 3)
    dx = 1.0 / n
    dt = 0.2 * dx * dx / 1.5

    def J(a, b):
        return 0.5 * ((heat_solve(a, b, steps, dt, dx, 64) - target) ** 2).sum().item()

    x = u0.clone().requires_grad_(True)
    y = alpha.clone().requires_grad_(True)
    (0.5 * ((heat_solve(x, y, steps, dt, dx, 64) - target) ** 2).sum()).backward()
    gen = torch.Generator(device="cuda").manual_seed(0)
    for _ in range(4):
        du = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=gen)
        da = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=gen)
        du /= du.norm()
        da /= da.norm()
        fd_u = (J(u0 + h * du, alpha) - J(u0 - h * du, alpha)) / (2 * h)
        fd_a = (J(u0, alpha + h * da) - J(u0, alpha - h * da)) / (2 * h)
        an_u = (x.grad * du).sum().item()
        an_a = (y.grad * da).sum().item()
        assert abs(fd_u - an_u) <= 1e-6 * max(abs(an_u), 1e-3), (fd_u, an_u)
        assert abs(fd_a - an_a) <= 1e-6 * max(abs(an_a), 1e-3), (fd_a, an_a)
