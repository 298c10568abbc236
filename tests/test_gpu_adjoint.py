"""GPU checks of the hand-written adjoint (mhd_adj_* of the C ABI).

* against the FP64 reference adjoint: PyTorch autograd through the CPU restatement of the step
  (oracle/torch_step.py, pinned to the C oracle by tests/test_torch_reference.py; its implicit
  solves are exact dense solves): the explicit-rate VJP, one step's VJP (state and eta) and a
  checkpointed multi-step trajectory, to 1e-9 relative L-infinity per field;
* against central finite differences of the GPU forward: dL/deta and the directional derivative
  along a smooth perturbation of the initial vector potential Az, through the torch.autograd
  binding, to 1e-6 relative, in a smooth pre-shock regime.
"""
import numpy as np
import pytest
import torch

from oracle import torch_step as ts
from tests_helpers import smooth_state

pytestmark = pytest.mark.gpu

REF_TOL = 1e-9


@pytest.fixture(scope="module")
def m():
    assert torch.cuda.is_available()
    import magnetohydrodynamics_simulator_b200 as mod

    assert mod.device_available(), "libmhd_b200.so has no kernels for this device"
    return mod


def _ptrs(t):
    return [t[k].data_ptr() for k in range(6)]


def _rel(got, want):
    """Per-field relative L-infinity, floor: the largest field magnitude of want."""
    floor = max(float(w.abs().max()) for w in want)
    return max(float((g - w).abs().max()) / max(float(w.abs().max()), 1e-3 * floor)
               for g, w in zip(got, want))


def _setup(nx, ny, seed, v_amp=0.3):
    dx, dy = 2 * np.pi / nx, 2 * np.pi / ny
    ic = smooth_state(nx, ny, dx, dy, seed, v_amp=v_amp)
    return dx, dy, torch.tensor(np.stack(ic))


def test_rate_vjp_matches_autograd(m):
    nx, ny = 24, 20
    dx, dy, U = _setup(nx, ny, 5)
    gen = torch.Generator().manual_seed(1)
    w = torch.randn(6, ny, nx, generator=gen, dtype=torch.float64)
    Ut = [U[k].clone().requires_grad_(True) for k in range(6)]
    want = torch.autograd.grad(ts.explicit_rhs(Ut, dx, dy), Ut, grad_outputs=list(w))
    adj = m.Adjoint(nx, ny, dx, dy, 1e-2, 1e-3, 1)
    u_d, w_d = U.cuda().contiguous(), w.cuda().contiguous()
    out = torch.empty_like(u_d)
    adj.rate_vjp(_ptrs(u_d), _ptrs(w_d), _ptrs(out))
    err = _rel(list(out.cpu()), list(want))
    assert err <= REF_TOL, err


@pytest.mark.parametrize("eta,dt", [(5e-2, 2e-3), (1.0, 1e-3), (0.0, 2e-3)])
def test_step_vjp_matches_autograd(m, eta, dt):
    nx, ny = 24, 20
    dx, dy, U = _setup(nx, ny, 7)
    L = ts.laplacian_matrix(nx, ny, dx, dy)
    gen = torch.Generator().manual_seed(2)
    lam_next = torch.randn(6, ny, nx, generator=gen, dtype=torch.float64)
    Ut = [U[k].clone().requires_grad_(True) for k in range(6)]
    eta_t = torch.tensor(eta, dtype=torch.float64, requires_grad=True)
    out = ts.imex_step(Ut, dt, eta_t, dx, dy, L)
    grads = torch.autograd.grad(out, Ut + [eta_t], grad_outputs=list(lam_next))
    adj = m.Adjoint(nx, ny, dx, dy, eta, dt, 1)
    u_d, l_d = U.cuda().contiguous(), lam_next.cuda().contiguous()
    lam = torch.empty_like(u_d)
    geta = adj.step_vjp(_ptrs(u_d), _ptrs(l_d), _ptrs(lam))
    err = _rel(list(lam.cpu()), list(grads[:6]))
    assert err <= REF_TOL, err
    want_eta = float(grads[6])
    assert abs(geta - want_eta) <= REF_TOL * max(abs(want_eta), 1e-12), (geta, want_eta)


def test_checkpointed_trajectory_matches_autograd(m):
    nx, ny = 20, 16
    dx, dy, U = _setup(nx, ny, 9)
    eta, dt, nsteps = 2e-2, 2e-3, 5
    L = ts.laplacian_matrix(nx, ny, dx, dy)
    target = U[0] * 1.01
    Ut = [U[k].clone().requires_grad_(True) for k in range(6)]
    eta_t = torch.tensor(eta, dtype=torch.float64, requires_grad=True)
    X = Ut
    for _ in range(nsteps):
        X = ts.imex_step(X, dt, eta_t, dx, dy, L)
    loss = 0.5 * ((X[0] - target) ** 2).sum()
    grads = torch.autograd.grad(loss, Ut + [eta_t])
    from magnetohydrodynamics_simulator_b200.autograd import trajectory

    adj = m.Adjoint(nx, ny, dx, dy, eta, dt, nsteps, checkpoint_every=2)  # segments 2, 2, 1
    u_d = U.cuda().contiguous().requires_grad_(True)
    e_d = torch.tensor(eta, dtype=torch.float64, device="cuda", requires_grad=True)
    uT = trajectory(u_d, e_d, adj)
    ref_T = torch.stack([x.detach() for x in X])
    assert _rel(list(uT.detach().cpu()), list(ref_T)) <= 1e-12
    loss_d = 0.5 * ((uT[0] - target.cuda()) ** 2).sum()
    loss_d.backward()
    err = _rel(list(u_d.grad.cpu()), list(grads[:6]))
    assert err <= REF_TOL, err
    assert abs(float(e_d.grad) - float(grads[6])) <= REF_TOL * abs(float(grads[6]))


def _loss_fd_setup(m, n=48, nsteps=12, every=4):
    """Smooth pre-shock state from 4 Fourier modes (velocity amplitude 0.05, Az amplitude 0.1,
    rho = p = 1) on a small grid; target from the forward solver at 0.8 eta."""
    from magnetohydrodynamics_simulator_b200.autograd import state_from_potential, trajectory

    dx = 2 * np.pi / n
    rng = np.random.default_rng(4)
    x = np.arange(n) * dx
    X, Y = np.meshgrid(x, x)

    def modes(amp, shift):
        f = np.zeros((n, n))
        for _ in range(4):
            kx, ky = rng.integers(-3, 4, size=2)
            f += amp * rng.uniform(0.5, 1.0) * np.sin(kx * (X + shift) + ky * (Y + shift) + rng.uniform(0, 6.28))
        return torch.tensor(f, device="cuda")

    vx, vy = modes(0.05, dx / 2), modes(0.05, dx / 2)
    az0 = modes(0.1, 0.0)
    daz = modes(0.1, 0.0)  # perturbation direction
    one = torch.ones(n, n, dtype=torch.float64, device="cuda")
    eta, dt = 5e-3, 2e-3
    adj = m.Adjoint(n, n, dx, dx, eta, dt, nsteps, checkpoint_every=every)

    def u0_of(az):
        return state_from_potential(az, one, vx, vy, one, dx, dx).contiguous()

    def loss(az, eta_t, target):
        uT = trajectory(u0_of(az), eta_t, adj)
        return 0.5 * ((uT[0] - target) ** 2).sum()

    loss.u0_of, loss.adj = u0_of, adj

    with torch.no_grad():
        target = trajectory(u0_of(az0), torch.tensor(0.8 * eta, dtype=torch.float64, device="cuda"), adj)[0].clone()
    return loss, az0, daz, eta, target


def test_gradients_match_central_differences(m):
    """Central differences of the GPU forward, taken on the final state (the difference of two
    trajectories, contracted afterwards), which stays well conditioned for small steps:
    * dL/deta of the quadratic density loss, step 1e-3 eta: <= 1e-6 relative;
    * the directional derivative along a smooth Az perturbation of a linear functional <w, rho(T)>
      (the adjoint's dot-product test), step 1e-6 of the potential: <= 5e-6 relative.
    The scheme is only piecewise smooth: the HLL wave-speed min/max (HLL.hpp:140-141) and minmod
    (MUSCL.hpp:11-17) switch branches densely in a smooth flow, so central differences approach the
    derivative only as the step shrinks (measured at 1024^2: 8e-5 at 1e-4, 1.2e-6 at 3e-7) until
    roundoff takes over (on this 48^2 grid: 1.6e-6 at 1e-6, 5.7e-6 at 3e-7); the exactness of the
    adjoint is shown against autograd above."""
    from magnetohydrodynamics_simulator_b200.autograd import trajectory

    loss, az0, daz, eta, target = _loss_fd_setup(m)
    az = az0.clone().requires_grad_(True)
    eta_t = torch.tensor(eta, dtype=torch.float64, device="cuda", requires_grad=True)
    L0 = loss(az, eta_t, target)
    L0.backward()
    g_eta = float(eta_t.grad)
    u0_of, adj = loss.u0_of, loss.adj
    gen = torch.Generator(device="cuda").manual_seed(3)
    w = torch.randn(target.shape, generator=gen, dtype=torch.float64, device="cuda")
    az = az0.clone().requires_grad_(True)
    e0 = torch.tensor(eta, dtype=torch.float64, device="cuda")
    (trajectory(u0_of(az), e0, adj)[0] * w).sum().backward()
    g_dir = float((az.grad * daz).sum())
    with torch.no_grad():
        h = 1e-3 * eta
        rp = trajectory(u0_of(az0), e0 + h, adj)[0]
        rm = trajectory(u0_of(az0), e0 - h, adj)[0]
        fd_eta = float((((rp - rm) / (2 * h)) * ((rp + rm) / 2 - target)).sum())
        s = 1e-6
        rp = trajectory(u0_of(az0 + s * daz), e0, adj)[0]
        rm = trajectory(u0_of(az0 - s * daz), e0, adj)[0]
        fd_dir = float((((rp - rm) / (2 * s)) * w).sum())
    assert abs(g_eta - fd_eta) <= 1e-6 * abs(fd_eta), (g_eta, fd_eta)
    assert abs(g_dir - fd_dir) <= 5e-6 * abs(fd_dir), (g_dir, fd_dir)


def _configured_setup(m, recompute_solves=False):
    """The configured differentiable workload: 1024^2, 4 random Fourier modes (velocity amplitude
    0.05, Az amplitude 0.1, rho = p = 1), eta = 5e-3, 100 fixed steps of 1e-3, checkpoint every 10;
    loss 1/2 |rho(T) - rho_target|^2 with the target from the forward solver at eta = 4e-3."""
    from magnetohydrodynamics_simulator_b200.autograd import state_from_potential, trajectory

    n, nsteps, every, dt, eta = 1024, 100, 10, 1e-3, 5e-3
    dx = 2 * np.pi / n
    rng = np.random.default_rng(5)
    X, Y = np.meshgrid(np.arange(n) * dx, np.arange(n) * dx)

    def modes(amp, shift):
        f = np.zeros((n, n))
        for _ in range(4):
            kx, ky = rng.integers(-4, 5, size=2)
            f += amp * rng.uniform(0.5, 1.0) * np.sin(kx * (X + shift) + ky * (Y + shift) + rng.uniform(0, 2 * np.pi))
        return torch.tensor(f, device="cuda")

    vx, vy = modes(0.05, dx / 2), modes(0.05, dx / 2)
    az0, daz = modes(0.1, 0.0), modes(0.1, 0.0)
    one = torch.ones(n, n, dtype=torch.float64, device="cuda")
    adj = m.Adjoint(n, n, dx, dx, eta, dt, nsteps, checkpoint_every=every, recompute_solves=recompute_solves)

    def u0_of(az):
        return state_from_potential(az, one, vx, vy, one, dx, dx).contiguous()

    with torch.no_grad():
        target = trajectory(u0_of(az0), torch.tensor(0.8 * eta, dtype=torch.float64, device="cuda"), adj)[0].clone()
    return adj, u0_of, az0, daz, eta, target


def test_configured_loss_gradients_match_central_differences(m):
    """The configured loss's gradient along the initial Az and in eta against central differences
    of the GPU forward, <= 1e-6 relative. The differences are taken on the final density (two
    trajectories, contracted with the loss's derivative afterwards), steps 3e-7 (Az) and 1e-3 eta."""
    from magnetohydrodynamics_simulator_b200.autograd import trajectory

    adj, u0_of, az0, daz, eta, target = _configured_setup(m)
    az = az0.clone().requires_grad_(True)
    eta_t = torch.tensor(eta, dtype=torch.float64, device="cuda", requires_grad=True)
    uT = trajectory(u0_of(az), eta_t, adj)
    (0.5 * ((uT[0] - target) ** 2).sum()).backward()
    g_dir, g_eta = float((az.grad * daz).sum()), float(eta_t.grad)
    e0 = torch.tensor(eta, dtype=torch.float64, device="cuda")
    with torch.no_grad():
        s = 3e-7
        rp = trajectory(u0_of(az0 + s * daz), e0, adj)[0]
        rm = trajectory(u0_of(az0 - s * daz), e0, adj)[0]
        fd_dir = float((((rp - rm) / (2 * s)) * ((rp + rm) / 2 - target)).sum())
        h = 1e-3 * eta
        rp = trajectory(u0_of(az0), e0 + h, adj)[0]
        rm = trajectory(u0_of(az0), e0 - h, adj)[0]
        fd_eta = float((((rp - rm) / (2 * h)) * ((rp + rm) / 2 - target)).sum())
    adj.close()
    assert abs(g_dir - fd_dir) <= 1e-6 * abs(fd_dir), (g_dir, fd_dir)
    assert abs(g_eta - fd_eta) <= 1e-6 * abs(fd_eta), (g_eta, fd_eta)


def test_recomputed_solves_give_identical_gradients(m):
    """MHD_ADJ_RECOMPUTE_SOLVES (one segment's solutions kept, each segment re-solved in the
    backward pass) gives bit-identical gradients with fewer planes."""
    nx, ny = 40, 36
    dx, dy, U = _setup(nx, ny, 11)
    eta, dt, nsteps, every = 2e-2, 2e-3, 9, 3
    u_d = U.cuda().contiguous()
    gen = torch.Generator(device="cuda").manual_seed(4)
    gT = torch.randn(u_d.shape, generator=gen, dtype=torch.float64, device="cuda")
    outs = []
    for recompute in (False, True):
        adj = m.Adjoint(nx, ny, dx, dy, eta, dt, nsteps, checkpoint_every=every, recompute_solves=recompute)
        uT, g0 = torch.empty_like(u_d), torch.empty_like(u_d)
        torch.cuda.synchronize()
        adj.forward(_ptrs(u_d), _ptrs(uT))
        geta = adj.backward(_ptrs(gT), _ptrs(g0))
        outs.append((uT.cpu(), g0.cpu(), geta, adj.device_bytes))
        adj.close()
    (uA, gA, eA, bA), (uB, gB, eB, bB) = outs
    assert torch.equal(uA, uB) and torch.equal(gA, gB) and eA == eB
    # 2 * nsteps solution planes against 2 * every
    assert bA - bB == 2 * (nsteps - every) * nx * ny * 8, (bA, bB)
