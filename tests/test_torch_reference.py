"""CPU: the PyTorch FP64 restatement used as the reference adjoint (oracle/torch_step.py) computes
the same forward step as the C oracle, so its autograd gradients are those of the reference
algorithm."""
import numpy as np
import torch

from oracle import torch_step as ts
from oracle.oracle import Oracle, rel_linf
from tests_helpers import smooth_state


def test_explicit_rate_and_steps_match_oracle():
    nx, ny = 24, 20
    dx, dy = 2 * np.pi / nx, 2 * np.pi / ny
    eta, dt = 5e-2, 2e-3
    ic = smooth_state(nx, ny, dx, dy, 3)
    o = Oracle(nx, ny, dx, dy, eta)
    o.set_state(ic)
    U = [torch.tensor(f) for f in ic]
    for got, want in zip(ts.explicit_rhs(U, dx, dy), o.explicit_rhs()):
        assert rel_linf(got.numpy(), want, 1.0) <= 1e-14
    L = ts.laplacian_matrix(nx, ny, dx, dy)
    for _ in range(3):
        o.step(dt)
        U = ts.imex_step(U, dt, eta, dx, dy, L)
    for got, want in zip(U, o.get_state()):
        assert rel_linf(got.numpy(), want, 1.0) <= 1e-13


def test_state_from_potential_matches_package_builder():
    from magnetohydrodynamics_simulator_b200.autograd import state_from_potential

    nx, ny = 16, 12
    dx, dy = 2 * np.pi / nx, 2 * np.pi / ny
    rng = np.random.default_rng(0)
    az = torch.tensor(rng.standard_normal((ny, nx)))
    rho = torch.tensor(1.0 + 0.1 * rng.standard_normal((ny, nx)))
    vx, vy = (torch.tensor(0.1 * rng.standard_normal((ny, nx))) for _ in range(2))
    p = torch.ones(ny, nx, dtype=torch.float64)
    azc = torch.zeros(ny + 1, nx + 1, dtype=torch.float64)
    azc[:ny, :nx] = az
    azc[ny, :nx] = az[0]
    azc[:, nx] = azc[:, 0]
    want = ts.state_from_potential(azc, rho, vx, vy, p, dx, dy)
    got = state_from_potential(az, rho, vx, vy, p, dx, dy)
    for g, w in zip(got, want):
        assert torch.allclose(g, w, rtol=1e-15, atol=1e-15)
