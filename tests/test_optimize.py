"""Batched L-BFGS and the regularisers of the inverse-design loop -- CPU only
(torch tensors on the CPU run the same code the GPU path runs on device
tensors; tests/test_gpu_parity.py drives it with the GPU cost/gradient).

The regularisers restate scripts/lib/regularizers.jl and are checked by
known answers and central differences; the optimiser is checked on analytic
objectives against scipy's L-BFGS-B minimum.
"""
import math

import numpy as np
import pytest
import torch
from scipy.optimize import minimize

from fiberlab_gpu import optimize as OP
from fiberlab_gpu import problem as P


def _fd(f, x, d, h=1e-6):
    return (f(x + h * d) - f(x - h * d)) / (2 * h)


def test_gdd_penalty_known_answer_and_gradient():
    nt, dt, lam = 64, 0.05, 3e-4
    dw = 2 * math.pi / (nt * dt)
    a = 0.7
    centred = a * (torch.arange(nt, dtype=torch.float64) - nt // 2) ** 2
    phi = torch.fft.ifftshift(centred)
    J, _ = OP.gdd_penalty(phi, dt, lam)
    assert float(J) == pytest.approx(lam * (nt - 2) * (2 * a) ** 2 / dw ** 3, rel=1e-12)
    rng = np.random.default_rng(0)
    x = torch.from_numpy(rng.standard_normal((2, nt)))
    J, g = OP.gdd_penalty(x, dt, lam)
    d = torch.from_numpy(rng.standard_normal((2, nt)))
    fd = _fd(lambda y: OP.gdd_penalty(y, dt, lam)[0], x, d)
    assert torch.allclose(fd, torch.sum(g * d, dim=1), rtol=1e-6)
    J0, g0 = OP.gdd_penalty(x, dt, 0.0)
    assert torch.all(J0 == 0) and torch.all(g0 == 0)


def test_boundary_penalty_gradient_and_floor():
    rng = np.random.default_rng(1)
    nt, M = 64, 3
    u0 = torch.from_numpy(rng.standard_normal((M, nt)) + 1j * rng.standard_normal((M, nt)))
    phi = torch.from_numpy(0.3 * rng.standard_normal(nt))

    def J_of(p):
        return OP.boundary_phase_penalty(u0 * torch.exp(1j * p), 0.5, shared=True)[0]
    J, g = OP.boundary_phase_penalty(u0 * torch.exp(1j * phi), 0.5, shared=True)
    d = torch.from_numpy(rng.standard_normal(nt))
    assert float(_fd(J_of, phi, d)) == pytest.approx(float(torch.sum(g * d)), rel=1e-6)
    # per-mode phases: the shared gradient is the mode sum of the per-mode one
    Jm, gm = OP.boundary_phase_penalty(u0 * torch.exp(1j * phi), 0.5, shared=False)
    assert float(Jm) == pytest.approx(float(J)) and torch.allclose(gm.sum(dim=0), g)
    # a pulse confined to the middle of the window: below the floor, no penalty
    t = torch.arange(nt, dtype=torch.float64) - nt // 2
    centred = torch.fft.ifft(torch.exp(-(t / 2) ** 2).to(torch.complex128))
    Jc, gc = OP.boundary_phase_penalty(centred[None], 0.5)
    assert float(Jc) == 0.0 and torch.all(gc == 0)


def test_log_surface():
    J, g = OP.apply_log_surface(torch.tensor([1e-3, 0.0]), torch.ones((2, 3)))
    assert float(J[0]) == pytest.approx(-30.0)
    assert float(J[1]) == pytest.approx(-150.0)
    assert float(g[0, 0]) == pytest.approx(10 / (math.log(10) * 1e-3))


def _rosenbrock(x):
    a, b = x[:, :-1], x[:, 1:]
    J = torch.sum(100 * (b - a * a) ** 2 + (1 - a) ** 2, dim=1)
    g = torch.zeros_like(x)
    g[:, :-1] += -400 * a * (b - a * a) - 2 * (1 - a)
    g[:, 1:] += 200 * (b - a * a)
    return J, g


def test_lbfgs_rosenbrock_batch_matches_scipy():
    rng = np.random.default_rng(2)
    x0 = torch.from_numpy(rng.uniform(-1.5, 1.5, (4, 10)))
    res = OP.lbfgs(_rosenbrock, x0, max_iter=300, f_abstol=0.0, g_abstol=1e-7)
    for b in range(4):
        ref = minimize(lambda v: float(_rosenbrock(torch.from_numpy(v[None]))[0][0]),
                       x0[b].numpy(), jac=lambda v: _rosenbrock(torch.from_numpy(v[None]))[1][0].numpy(),
                       method="L-BFGS-B", options={"maxiter": 2000, "gtol": 1e-10, "ftol": 0})
        # the same minimum as scipy from the same start (the global one, or
        # the extended Rosenbrock's local minimum near x1 = -1 at J = 3.98658)
        assert float(res.J[b]) == pytest.approx(ref.fun, abs=1e-8)
        assert np.allclose(res.x[b].numpy(), ref.x, atol=1e-4)
        assert res.status[b] in ("converged_g", "converged_f")
    # every accepted step decreased the cost (Armijo)
    tr = torch.stack(res.trace)
    assert torch.all(tr[1:] <= tr[:-1] + 1e-12)
    assert res.evaluations >= res.iterations.max() + 1


def test_lbfgs_quadratic_exact_and_stopping():
    rng = np.random.default_rng(3)
    Q = rng.standard_normal((8, 8))
    A = torch.from_numpy(Q @ Q.T + 8 * np.eye(8))
    c = torch.from_numpy(rng.standard_normal(8))

    def fg(x):
        Ax = x @ A
        return 0.5 * torch.sum(x * Ax, dim=1) - x @ c, Ax - c
    xstar = torch.linalg.solve(A, c)
    res = OP.lbfgs(fg, torch.zeros((2, 8), dtype=torch.float64), max_iter=100, f_abstol=None,
                   g_abstol=1e-10)
    assert torch.allclose(res.x, xstar[None].expand(2, 8), atol=1e-8)
    assert res.status == ["converged_g", "converged_g"]
    one = OP.lbfgs(fg, torch.zeros((1, 8), dtype=torch.float64), max_iter=1)
    assert one.status == ["max_iter"] and one.iterations[0] == 1
    with pytest.raises(P.ArgumentError):
        OP.lbfgs(fg, torch.zeros((1, 8)), max_iter=0)
