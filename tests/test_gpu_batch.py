"""GPU parity of the batched step (mhd_batch_* of the C ABI) against the CPU oracle and against
single-instance contexts.

Every instance of a batch must get the step it would get alone: its own CFL dt, its own matrix
coefficient, its own CG convergence. The batch sums each CG reduction in another fixed order than
a single context, so the two agree to rounding (not bit for bit); the explicit stages are
bit-identical. Tolerances: 1e-12 relative L-infinity per field for a few steps against the oracle
(near-zero fields against a floor of 1), 1e-10 for longer runs, CG products within 1.
"""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, default_alpha, rel_linf
from tests_helpers import smooth_state

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


# (nx, ny, eta, ct_mode, seed): uneven sizes, dx != dy, eta = 0 (vanishing right-hand side),
# a 2x2 grid, both CT modes
SPECS = [
    (40, 24, 5e-2, 0, 1),
    (33, 17, 0.0, 0, 2),
    (64, 48, 1.0, 1, 3),
    (2, 2, 1e-2, 0, 4),
    (31, 70, 3e-3, 0, 5),
    (96, 96, 1e-3, 0, 6),
]


def _instances(specs):
    out = []
    for nx, ny, eta, ct, seed in specs:
        dx, dy = 2 * np.pi / nx, 2 * np.pi / ny
        out.append(dict(nx=nx, ny=ny, dx=dx, dy=dy, eta=eta, ct_mode=ct,
                        ic=smooth_state(nx, ny, dx, dy, seed)))
    return out


def _batch(m, insts):
    b = m.Batch([{k: v for k, v in s.items() if k != "ic"} for s in insts])
    for i, s in enumerate(insts):
        b.set_state(i, s["ic"])
    return b


def _oracle(s):
    o = Oracle(s["nx"], s["ny"], s["dx"], s["dy"], s["eta"], ct_abs_mode=s["ct_mode"])
    o.set_state(s["ic"])
    return o


def _max_err(got, want, floor=1.0):
    return max(rel_linf(g, w, floor) for g, w in zip(got, want))


def test_batch_cfl_steps_match_oracle(m):
    insts = _instances(SPECS)
    b = _batch(m, insts)
    orcs = [_oracle(s) for s in insts]
    for _ in range(3):
        dts = []
        for i, o in enumerate(orcs):
            dt = o.cfl_dt()
            assert abs(b.cfl_dt(i) - dt) <= 1e-13 * dt
            dts.append(dt)
        b.step()  # every instance takes its own CFL step on the device
        b.synchronize()
        prods = b.last_cg_products()
        for i, o in enumerate(orcs):
            p_orc = o.step(dts[i])
            assert all(abs(int(a) - int(c)) <= 1 for a, c in zip(prods[i], p_orc)), (i, prods[i], p_orc)
    for i, o in enumerate(orcs):
        err = _max_err(b.get_state(i), o.get_state())
        assert err <= STEP_TOL, (i, err)
        assert b.divb(i)[1] <= 1e-12


def test_batch_given_dts_and_fixed_coefficient(m):
    insts = _instances(SPECS[:4])
    b = _batch(m, insts)
    b.set_implicit_coefficient(2, 7.5e-3)
    dts = [1e-3, 2e-3, 5e-4, 1e-3]
    b.step(dts)
    b.synchronize()
    for i, s in enumerate(insts):
        o = _oracle(s)
        alpha = 7.5e-3 if i == 2 else default_alpha(dts[i], s["eta"])
        o.step(dts[i], alpha=alpha)
        err = _max_err(b.get_state(i), o.get_state())
        assert err <= STEP_TOL, (i, err)


def test_batch_run_matches_single_contexts(m):
    insts = _instances(SPECS)
    b = _batch(m, insts)
    nsteps = 9  # four graph replays of two steps, then one plain step
    dts_b, prods_b = b.run(nsteps)
    b.synchronize()
    for i, s in enumerate(insts):
        ctx = m.Context(s["nx"], s["ny"], s["dx"], s["dy"], s["eta"], ct_mode=s["ct_mode"])
        ctx.set_state(s["ic"])
        dts_c, prods_c = ctx.run(nsteps)
        ctx.synchronize()
        np.testing.assert_allclose(dts_b[i], dts_c, rtol=1e-12, atol=0)
        assert np.abs(prods_b[i] - prods_c).max() <= 1, (i, prods_b[i], prods_c)
        err = _max_err(b.get_state(i), ctx.get_state())
        assert err <= RUN_TOL, (i, err)


def test_batch_run_matches_oracle_driver(m):
    """The batched driver loop against the oracle stepped with the same dts and the driver's
    matrix rule (integrator_main.cpp:55-60, 87-95)."""
    insts = _instances(SPECS[:3])
    b = _batch(m, insts)
    nsteps = 6
    dts_b, _ = b.run(nsteps)
    b.synchronize()
    g = (2.0 - np.sqrt(2.0)) / 2.0
    for i, s in enumerate(insts):
        o = _oracle(s)
        alpha = None
        prev = None
        for k in range(nsteps):
            dt = o.cfl_dt()
            assert abs(dts_b[i][k] - dt) <= 1e-12 * dt, (i, k, dts_b[i][k], dt)
            if alpha is None:
                alpha, prev = (dt * s["eta"]) * g, dt
            if s["eta"] > 0 and abs(dt - prev) > 1e-10 * dt:
                alpha = (dt * s["eta"]) * g
            prev = dt
            o.step(dt, alpha=alpha)
        err = _max_err(b.get_state(i), o.get_state())
        assert err <= RUN_TOL, (i, err)


def test_graph_replay_equals_plain_launches(m):
    insts = _instances(SPECS[:4])
    b1 = _batch(m, insts)
    b2 = _batch(m, insts)
    d1, p1 = b1.run(6)
    os.environ["MHD_B200_NO_GRAPH"] = "1"
    try:
        d2, p2 = b2.run(6)
    finally:
        del os.environ["MHD_B200_NO_GRAPH"]
    assert np.array_equal(d1, d2) and np.array_equal(p1, p2)
    for i in range(len(insts)):
        for f1, f2 in zip(b1.get_state(i), b2.get_state(i)):
            assert np.array_equal(f1, f2)


def test_more_instances_than_one_solver_launch(m):
    """70 instances: the implicit solves take two launches (64 + 6 instances)."""
    rng = np.random.default_rng(11)
    specs = [(int(rng.integers(6, 20)), int(rng.integers(6, 20)), float(10 ** rng.uniform(-3, -1)), 0,
              100 + k) for k in range(70)]
    insts = _instances(specs)
    b = _batch(m, insts)
    assert b.launches_per_step == 8
    dts = np.array([5e-4] * len(insts))
    for _ in range(2):
        b.step(dts)
    b.synchronize()
    for i, s in enumerate(insts):
        o = _oracle(s)
        for _ in range(2):
            o.step(5e-4)
        err = _max_err(b.get_state(i), o.get_state())
        assert err <= STEP_TOL, (i, err)


def test_autotune_restores_state_and_keeps_parity(m):
    insts = _instances(SPECS)
    b = _batch(m, insts)
    before = [b.get_state(i) for i in range(len(insts))]
    cfl_before = [b.cfl_dt(i) for i in range(len(insts))]
    t = b.autotune()
    assert t["stage_rows"] >= 1 and t["cg_order"] in (0, 1)
    assert t["cg_rows"] >= 1 or (t["cg_rows"] == 0 and t["cg_order"] == 1)  # 0: heights per phase
    assert t["stage_ms"] > 0 and t["cg_ms"] > 0
    for i in range(len(insts)):
        for f0, f1 in zip(before[i], b.get_state(i)):
            assert np.array_equal(f0, f1)
        assert b.cfl_dt(i) == cfl_before[i]
    b.run(4)
    b.synchronize()
    for i, s in enumerate(insts):
        ctx = m.Context(s["nx"], s["ny"], s["dx"], s["dy"], s["eta"], ct_mode=s["ct_mode"])
        ctx.set_state(s["ic"])
        ctx.run(4)
        err = _max_err(b.get_state(i), ctx.get_state())
        assert err <= RUN_TOL, (i, err)


@pytest.mark.parametrize("stage_rows,cg_rows,cg_order,tail", [(1, 1, 0, 0), (7, 3, 1, 0), (300, 300, 0, 0),
                                                            (16, 8, 0, 5), (64, 32, 1, 3), (48, 0, 1, 0)])
def test_every_decomposition_gives_the_same_step(m, stage_rows, cg_rows, cg_order, tail):
    insts = _instances(SPECS)
    b = _batch(m, insts)
    b.set_tuning(stage_rows, cg_rows, cg_order, tail)
    assert b.tuning()["stage_tail_rows"] == tail
    dts = [1e-3] * len(insts)
    b.step(dts)
    b.synchronize()
    for i, s in enumerate(insts):
        o = _oracle(s)
        o.step(1e-3)
        err = _max_err(b.get_state(i), o.get_state())
        assert err <= STEP_TOL, (i, err)


def test_phase_chosen_tile_height_needs_tiles(m):
    """cg_rows = 0 (a tile height chosen phase by phase) exists for the tile order only."""
    b = _batch(m, _instances(SPECS[:2]))
    with pytest.raises(m.MHDError):
        b.set_tuning(64, 0, 0, 0)
    b.set_tuning(64, 0, 1, 0)
    assert b.tuning()["cg_rows"] == 0


def test_nonfinite_instance_is_reported_alone(m):
    insts = _instances(SPECS[:3])
    insts[1]["ic"] = [f.copy() for f in insts[1]["ic"]]
    insts[1]["ic"][0][3, 5] = np.nan
    b = _batch(m, insts)
    b.step([1e-3, 1e-3, 1e-3])
    worst, per = b.synchronize_status()
    assert per[1] == 3 and per[0] == 0 and per[2] == 0, per
    assert worst == 3
    worst2, per2 = b.synchronize_status()  # cleared
    assert worst2 == 0 and per2 == [0, 0, 0]


def test_sine_wave_batch_decays_analytically(m):
    """Decaying magnetic sine waves of several sizes and resistivities in one batch: each
    amplitude follows the implicit scheme's own decay factor per step (benchmarks.hpp:352-417)."""
    cases = [(64, 0.5), (96, 2.0), (128, 10.0)]
    insts = []
    for n, eta in cases:
        dx = 2 * np.pi / n
        o = Oracle(n, n, dx, dx, eta)
        o.init_sine_wave(az_amp=1e-3, kx=1.0, ky=1.0, use_sin=True)
        insts.append(dict(nx=n, ny=n, dx=dx, dy=dx, eta=eta, ct_mode=0, ic=o.get_state()))
    b = _batch(m, insts)
    dt, nsteps = 1e-3, 20
    b.run(nsteps, dt_fixed=dt)
    b.synchronize()
    for i, (n, eta) in enumerate(cases):
        s = insts[i]
        o = _oracle(s)
        for _ in range(nsteps):
            o.step(dt)
        got, want = b.get_state(i), o.get_state()
        assert rel_linf(got[4], want[4]) <= RUN_TOL and rel_linf(got[5], want[5]) <= RUN_TOL
        amp0 = np.abs(s["ic"][4]).max()
        ratio = np.abs(got[4]).max() / amp0
        exact = np.exp(-eta * 2.0 * nsteps * dt)
        assert abs(ratio - exact) <= 2e-3 * exact, (n, eta, ratio, exact)
