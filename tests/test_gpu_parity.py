"""GPU parity of the IMEX step against the CPU oracle and the reference's golden vectors.

Every test calls the product through the C ABI (libmhd_b200.so via ctypes). Tolerances:
* one or a few steps on small grids: 1e-12 relative L-infinity per field (the oracle is strict
  IEEE, the GPU contracts FMAs and sums reductions in another order; measured differences are
  ~1e-15);
* long runs (Orszag-Tang 128^2, 200 steps): 1e-10 relative L-infinity per field, the product bar;
* |div B|_inf <= 1e-12 after every run.
Near-zero fields are compared against a stated floor (rel_linf's `floor`).
"""
import numpy as np
import pytest

from conftest import fields, load_golden
from oracle.oracle import Oracle, default_alpha, rel_linf

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-12
RUN_TOL = 1e-10


@pytest.fixture(scope="module")
def m():
    import torch

    assert torch.cuda.is_available()
    import magnetohydrodynamics_simulator_b200 as mod

    assert mod.device_available(), "libmhd_b200.so has no kernels for this device"
    return mod


def _errs(got, want, floor=0.0):
    return [rel_linf(g, w, floor) for g, w in zip(got, want)]


def _pair(m, nx, ny, dx, dy, eta, ic, **kw):
    orc = Oracle(nx, ny, dx, dy, eta, ct_abs_mode=kw.get("ct_mode", 0))
    orc.set_state(ic)
    ctx = m.Context(nx, ny, dx, dy, eta, **kw)
    ctx.set_state(ic)
    return orc, ctx


@pytest.mark.parametrize("eta", [0.0, 1e-3, 0.5])
def test_one_step_orszag_tang(m, eta):
    n = 32
    dx = m.problems.grid_spacing(n)
    orc = Oracle(n, n, dx, dx, eta)
    orc.init_orszag_tang()
    ic = orc.get_state()
    ctx = m.Context(n, n, dx, dx, eta)
    ctx.set_state(ic)
    dt = orc.cfl_dt()
    assert abs(ctx.cfl_dt() - dt) <= 1e-14 * dt
    ctx.step(dt)
    ctx.synchronize()
    p_orc = orc.step(dt)
    errs = _errs(ctx.get_state(), orc.get_state(), floor=1.0)
    assert max(errs) <= STEP_TOL, errs
    p_gpu = ctx.last_cg_products()
    assert all(abs(a - b) <= 1 for a, b in zip(p_gpu, p_orc)), (p_gpu, p_orc)


def test_non_square_random_state_matches_reference(m):
    d = load_golden("random40x24_ref.npz")
    nx, ny, dx, dy, eta = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"]), float(d["eta"])
    ctx = m.Context(nx, ny, dx, dy, eta)
    ctx.set_state(fields(d, "ic"))
    for dt in d["dts"]:
        ctx.step(float(dt))
    ctx.synchronize()
    errs = _errs(ctx.get_state(), fields(d, "final"))
    assert max(errs) <= STEP_TOL, errs


def test_upwind_branch_matches_reference(m):
    """Corner velocities above 1 take the upwind branch of the (int-truncated) CT test."""
    d = load_golden("upwind32_ref.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    ctx = m.Context(nx, ny, dx, dy, float(d["eta"]))
    ctx.set_state(fields(d, "ic"))
    assert abs(ctx.cfl_dt() - d["dts"][0]) <= 1e-14 * d["dts"][0]
    for dt in d["dts"]:
        ctx.step(float(dt))
    ctx.synchronize()
    errs = _errs(ctx.get_state(), fields(d, "final"))
    assert max(errs) <= STEP_TOL, errs


def test_true_abs_mode_matches_oracle(m):
    n = 32
    dx = m.problems.grid_spacing(n)
    orc = Oracle(n, n, dx, dx, 1e-3, ct_abs_mode=1)
    orc.init_orszag_tang()
    ic = orc.get_state()
    ctx = m.Context(n, n, dx, dx, 1e-3, ct_mode=m.CT_TRUE_ABS)
    ctx.set_state(ic)
    for _ in range(3):
        dt = orc.cfl_dt()
        orc.step(dt)
        ctx.step(dt)
    ctx.synchronize()
    errs = _errs(ctx.get_state(), orc.get_state(), floor=1.0)
    assert max(errs) <= STEP_TOL, errs


def test_orszag_tang_128_200_steps_matches_reference(m):
    """The CPU-runnable configuration: 128^2, eta = 1e-3, the reference driver's dt sequence."""
    d = load_golden("ot128_ref.npz")
    n, dx, eta = int(d["nx"]), float(d["dx"]), float(d["eta"])
    orc = Oracle(n, n, dx, dx, eta)
    orc.init_orszag_tang()
    ctx = m.Context(n, n, dx, dx, eta)
    ctx.set_state(orc.get_state())
    prods = []
    for dt in d["dts"]:
        ctx.step(float(dt))
    ctx.synchronize()
    errs = _errs(ctx.get_state(), fields(d, "final"))
    assert max(errs) <= RUN_TOL, errs
    rms, mx = ctx.divb()
    assert mx <= 1e-12, mx
    # the reference's own value at the same point, for the record
    assert abs(mx - d["divb"][1]) <= 1e-12


def test_driver_loop_on_device_matches_reference(m):
    """mhd_run: dynamic CFL dt and matrix regeneration on the device, CUDA-graph replayed."""
    d = load_golden("ot128_ref.npz")
    n, dx, eta = int(d["nx"]), float(d["dx"]), float(d["eta"])
    orc = Oracle(n, n, dx, dx, eta)
    orc.init_orszag_tang()
    ctx = m.Context(n, n, dx, dx, eta)
    ctx.set_state(orc.get_state())
    dts, prods = ctx.run(int(d["steps"]))
    ctx.synchronize()
    assert np.max(np.abs(dts - d["dts"]) / d["dts"]) <= 1e-12
    assert np.max(np.abs(prods - d["cg_products"])) <= 1
    errs = _errs(ctx.get_state(), fields(d, "final"))
    assert max(errs) <= RUN_TOL, errs


def test_run_equals_repeated_steps(m):
    n = 48
    dx = m.problems.grid_spacing(n)
    ic = m.problems.orszag_tang(n, n, dx, dx)
    a = m.Context(n, n, dx, dx, 1e-2)
    b = m.Context(n, n, dx, dx, 1e-2)
    a.set_state(ic)
    b.set_state(ic)
    dt = 2e-3
    a.run(9, dt_fixed=dt, record=False)
    for _ in range(9):
        b.step(dt)
    a.synchronize()
    b.synchronize()
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)


def test_decaying_wave_matches_reference(m):
    d = load_golden("dsw64_ref.npz")
    n, dx, eta = int(d["nx"]), float(d["dx"]), float(d["eta"])
    ctx = m.Context(n, n, dx, dx, eta)
    ctx.set_state(fields(d, "ic"))
    for dt in d["dts"]:
        ctx.step(float(dt))
    ctx.synchronize()
    # momenta are O(1e-9) Lorentz-driven: compare at the B0^2 = 1e-6 scale (see oracle tests)
    errs = _errs(ctx.get_state(), fields(d, "final"), floor=1e-6)
    assert max(errs) <= RUN_TOL, errs


def test_decaying_wave_512_matches_oracle(m):
    """Configured decaying wave at its full 512^2 size (eta = 10, dt = 1e-4), a few steps
    against the oracle: the CG-dominated path (tens of products per solve)."""
    n, eta, dt, steps = 512, 10.0, 1e-4, 3
    ic, dx = m.problems.sine_wave_config(n)
    orc, ctx = _pair(m, n, n, dx, dx, eta, ic)
    p_orc = [orc.step(dt) for _ in range(steps)]
    _, prods = ctx.run(steps, dt_fixed=dt)
    ctx.synchronize()
    errs = _errs(ctx.get_state(), orc.get_state(), floor=1e-6)
    assert max(errs) <= RUN_TOL, errs
    assert np.max(np.abs(prods - np.array(p_orc))) <= 1
    assert prods.min() > 30


def test_decaying_wave_512_analytic_decay(m):
    """Configured decaying wave: 512^2, eta = 10, dt = 1e-4, 100 steps.

    B is a single Fourier mode of the staggered Laplacian (eigenvalue lam), and the implicit
    part multiplies it by the ARS(2,2,2) (L-stable SDIRK2) amplification factor R(z),
    z = -eta*lam*dt, each step. The explicit part adds the HLL flux's numerical diffusion of the
    tangential field (order c_f * dx^3 * k^4 * t ~ 3e-7 relative here, the same in the
    reference), so: R(z)^n to 1e-6, exp(-eta*lam*t) to 2e-6 (plus the scheme's O(dt^2) error)
    and the continuous exp(-2 eta t) to 2e-5 (the grid's O(dx^2) error).
    """
    n, eta, dt, steps = 512, 10.0, 1e-4, 100
    ic, dx = m.problems.sine_wave_config(n)
    ctx = m.Context(n, n, dx, dx, eta)
    ctx.set_state(ic)
    dts, prods = ctx.run(steps, dt_fixed=dt)
    ctx.synchronize()
    s = ctx.get_state()
    amp = float(np.sum(s[5] * ic[5]) / np.sum(ic[5] * ic[5]))
    lam = 2 * (4.0 / dx**2) * np.sin(dx / 2) ** 2
    z = -eta * lam * dt
    g = (2.0 - np.sqrt(2.0)) / 2.0
    y1 = 1.0 / (1.0 - g * z)
    R = (1.0 + (1.0 - g) * z * y1) / (1.0 - g * z)
    t = steps * dt
    assert abs(amp - R**steps) <= 1e-6 * R**steps, (amp, R**steps)
    assert abs(amp - np.exp(-eta * lam * t)) <= 2e-6 * np.exp(-eta * lam * t)
    assert abs(amp - np.exp(-2 * eta * t)) <= 2e-5 * np.exp(-2 * eta * t)
    rms, mx = ctx.divb()
    assert mx <= 1e-12
    assert prods.min() > 30  # the CG-dominated configuration


def test_orszag_tang_point_symmetry(m):
    """OT is symmetric under (x, y) -> (-x, -y): rho, E, p even; v, B odd
    (scripts/OrszagTangInversionSymmetryDisplay.py:34-75, on cell centres)."""
    n = 128
    dx = m.problems.grid_spacing(n)
    orc = Oracle(n, n, dx, dx, 1e-3)
    orc.init_orszag_tang()
    ctx = m.Context(n, n, dx, dx, 1e-3)
    ctx.set_state(orc.get_state())
    ctx.run(100)
    ctx.synchronize()
    pr = ctx.primitives()

    def refl(a):  # cell (i, j) -> (N-1-i, N-1-j)
        return a[::-1, ::-1]

    scale = {k: max(np.max(np.abs(v)), 1.0) for k, v in pr.items()}
    for k in ("rho", "p"):
        assert np.max(np.abs(pr[k] - refl(pr[k]))) <= 1e-10 * scale[k], k
    for k in ("vx", "vy"):
        assert np.max(np.abs(pr[k] + refl(pr[k]))) <= 1e-10 * scale[k], k
    # cell-centred B of the point-reflected cell (faces reflect onto faces of the mirrored cell)
    for k in ("bxc", "byc"):
        assert np.max(np.abs(pr[k] + refl(pr[k]))) <= 1e-10 * scale[k], k


def test_resistive_rate_matches_reference(m):
    """resistive_B_term on device arrays: implicit rate against the reference's own (golden) solve,
    explicit rate against the oracle."""
    import torch

    d = load_golden("random40x24_ref.npz")
    nx, ny, dx, dy, eta = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"]), float(d["eta"])
    ctx = m.Context(nx, ny, dx, dy, eta)
    bxf = torch.tensor(d["ic_bxf"], device="cuda")
    byf = torch.tensor(d["ic_byf"], device="cuda")
    bx = torch.empty_like(bxf)
    by = torch.empty_like(byf)
    torch.cuda.synchronize()
    prods = ctx.resistive_rate(bxf.data_ptr(), byf.data_ptr(), bx.data_ptr(), by.data_ptr(),
                               solve_implicitly=True, alpha=float(d["implicit_alpha"]))
    ctx.synchronize()
    assert prods > 0
    errs = _errs([bx.cpu().numpy(), by.cpu().numpy()], [d["implicit_bx"], d["implicit_by"]])
    assert max(errs) <= STEP_TOL, errs
    # explicit
    orc = Oracle(nx, ny, dx, dy, eta)
    want_x = np.zeros((ny, nx))
    want_y = np.zeros((ny, nx))
    import ctypes
    from oracle.oracle import _ptr

    ic = [np.ascontiguousarray(d["ic_bxf"]), np.ascontiguousarray(d["ic_byf"])]
    orc.lib.orc_resistive_rate(ctypes.byref(orc.p), _ptr(ic[0]), _ptr(ic[1]), -1.0, _ptr(want_x), _ptr(want_y))
    assert ctx.resistive_rate(bxf.data_ptr(), byf.data_ptr(), bx.data_ptr(), by.data_ptr(),
                              solve_implicitly=False) == 0
    ctx.synchronize()
    errs = _errs([bx.cpu().numpy(), by.cpu().numpy()], [want_x, want_y])
    assert max(errs) <= STEP_TOL, errs


def test_cfl_primitives_and_divb_match_oracle(m):
    d = load_golden("random40x24_ref.npz")
    nx, ny, dx, dy, eta = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"]), float(d["eta"])
    orc, ctx = _pair(m, nx, ny, dx, dy, eta, fields(d, "ic"), courant=0.4)
    assert abs(ctx.cfl_dt() - orc.cfl_dt(0.4, 0.9)) <= 1e-14 * orc.cfl_dt(0.4, 0.9)
    pg, po = ctx.primitives(), orc.primitives()
    for k in po:
        assert rel_linf(pg[k], po[k], 1.0) <= 1e-14, k
    rms_g, mx_g = ctx.divb()
    rms_o, mx_o = orc.divb()
    assert abs(mx_g - mx_o) <= 1e-14 and abs(rms_g - rms_o) <= 1e-14


def test_padded_layout_round_trip(m):
    n, ng = 20, 2
    dx = m.problems.grid_spacing(n)
    ic = m.problems.orszag_tang(n, n, dx, dx)
    padded = []
    for f in ic:
        p = np.full((n + 2 * ng, n + 2 * ng), -7.0)
        p[ng:-ng, ng:-ng] = f
        padded.append(p)
    ctx = m.Context(n, n, dx, dx, 0.0)
    ctx.set_state(padded, layout=m.LAYOUT_PADDED, ng=ng)
    dense = ctx.get_state()
    for a, b in zip(dense, ic):
        assert np.array_equal(a, b)
    back = ctx.get_state(layout=m.LAYOUT_PADDED, ng=ng)
    for a, b in zip(back, ic):
        assert np.array_equal(a, np.pad(b, ng, mode="wrap"))  # ghosts = periodic copies


def test_nonfinite_state_is_reported(m):
    n = 32
    dx = m.problems.grid_spacing(n)
    ic = m.problems.orszag_tang(n, n, dx, dx)
    ic[3][5, 7] = np.nan
    ctx = m.Context(n, n, dx, dx, 1e-3)
    ctx.set_state(ic)
    ctx.step(1e-3)
    assert ctx.synchronize_status() == 3  # MHD_ERR_NONFINITE
    assert ctx.synchronize_status() == 0  # the status is cleared once read


def test_cg_iteration_cap_is_reported(m):
    ic, dx = m.problems.sine_wave_config(64)
    ctx = m.Context(64, 64, dx, dx, 10.0, cg_max_iters=2)
    ctx.set_state(ic)
    ctx.step(1e-4)
    assert ctx.synchronize_status() == 4  # MHD_ERR_CG_NOT_CONVERGED
    assert ctx.last_cg_products() == (2, 2)


def test_cg_wait_limit_returns_timeout(m):
    """A grid-wide wait of the persistent CG that runs out of time ends the kernel with a
    status instead of spinning: a 1 microsecond limit on a 1024^2 solve always runs out."""
    ic, dx = m.problems.sine_wave_config(1024)
    ctx = m.Context(1024, 1024, dx, dx, 10.0, cg_timeout_s=1e-6)
    ctx.set_state(ic)
    ctx.step(1e-4)
    assert ctx.synchronize_status() == 5  # MHD_ERR_TIMEOUT
    # the context stays usable
    ctx2 = m.Context(64, 64, 2 * np.pi / 64, 2 * np.pi / 64, 1.0)
    ic2, _ = m.problems.sine_wave_config(64)
    ctx2.set_state(ic2)
    ctx2.step(1e-4)
    assert ctx2.synchronize_status() == 0


def test_zero_resistivity_skips_solves(m):
    n = 32
    dx = m.problems.grid_spacing(n)
    ctx = m.Context(n, n, dx, dx, 0.0)
    ctx.set_state(m.problems.orszag_tang(n, n, dx, dx))
    ctx.step(1e-3)
    ctx.synchronize()
    assert ctx.last_cg_products() == (0, 0)


@pytest.mark.parametrize("shape", [(2, 2), (3, 5), (33, 17), (70, 130)])
def test_small_and_ragged_grids(m, shape):
    """Sizes that are not multiples of any tile, down to the reference's minimum of 2 cells."""
    nx, ny = shape
    dx, dy = 2 * np.pi / nx, 1.3 * np.pi / ny
    from tests_helpers import smooth_state

    ic = smooth_state(nx, ny, dx, dy, seed=nx * 1000 + ny)
    orc, ctx = _pair(m, nx, ny, dx, dy, 0.05, ic)
    for _ in range(2):
        dt = 0.5 * orc.cfl_dt()
        orc.step(dt)
        ctx.step(dt)
    ctx.synchronize()
    errs = _errs(ctx.get_state(), orc.get_state(), floor=1.0)
    assert max(errs) <= STEP_TOL, errs


@pytest.mark.parametrize("name", ["alfven_wave", "gaussian_pulse", "acoustic_wave", "sausage", "kink"])
def test_other_initial_conditions_match_reference(m, name):
    """The reference's five other initial conditions (benchmarks.hpp:78-350), built by
    problems.py, through the device driver loop (5 CFL steps, eta = 5e-3) against the reference's
    own driver loop: the low-beta sausage pinch, the kink, the Gaussian pulse advected at |v| = 1.4,
    the Alfven and acoustic waves. Floor 1e-3: the fixtures' perturbation scale (m_x of the Alfven
    and acoustic waves vanishes in exact arithmetic)."""
    d = load_golden("fixtures32x24_ref.npz")
    nx, ny, dx, dy, eta = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"]), float(d["eta"])
    ctx = m.Context(nx, ny, dx, dy, eta)
    ctx.set_state(m.problems.FIXTURES[name](nx, ny, dx, dy))
    dts, prods = ctx.run(int(d["steps"]))
    ctx.synchronize()
    want_dts = d[f"{name}_dts"]
    assert np.max(np.abs(dts - want_dts) / want_dts) <= 1e-12
    assert np.max(np.abs(prods - d[f"{name}_cg_products"])) <= 1
    errs = _errs(ctx.get_state(), fields(d, f"{name}_final"), floor=1e-3)
    assert max(errs) <= STEP_TOL, errs
    assert ctx.divb()[1] <= 1e-12


def test_pipelined_host_transfers_match_synchronous_calls(m):
    """mhd_set_state_async / mhd_get_state_async (copies on two copy streams, a step's read-back
    overlapping the next upload) round-trip every step's state through pinned host planes and give
    the same states, bit for bit, as the synchronous set_state / get_state calls; the read-back
    also holds the state when no upload follows it."""
    import torch

    n = 96
    dx = m.problems.grid_spacing(n)
    ic = m.problems.orszag_tang(n, n, dx, dx)
    a = m.Context(n, n, dx, dx, 1e-2)
    b = m.Context(n, n, dx, dx, 1e-2)
    pinned = [torch.empty((n, n), dtype=torch.float64, pin_memory=True).numpy() for _ in range(6)]
    for k in range(6):
        pinned[k][...] = ic[k]
    host = [f.copy() for f in ic]
    for _ in range(4):
        a.set_state_async(pinned)
        a.step(0.0)
        a.get_state_async(pinned)
        b.set_state(host)
        b.step(0.0)
        host = b.get_state()
    a.transfers_wait()
    for x, y in zip(pinned, host):
        assert np.array_equal(x, y)
    # a read-back followed by more steps: the steps wait for the copies
    a.get_state_async(pinned)
    a.step(1e-3)
    a.step(1e-3)
    a.transfers_wait()
    for x, y in zip(pinned, host):
        assert np.array_equal(x, y)
    b.step(1e-3)
    b.step(1e-3)
    a.synchronize()
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
    assert a.synchronize_status() == 0
