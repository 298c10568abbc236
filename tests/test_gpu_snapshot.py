"""GPU checks of the snapshot writer (mhd_snapshot_* of the C ABI) against the reference's file
format: the file the reference's own write_data_to_binary_file (diagnostics.hpp:90-131) wrote for a
state (tests/golden/snapshot20x14_ref.npz), and the oracle's restatement of that writer (pinned to
the same file by tests/test_oracle_golden.py) for other grids and ghost widths.

Tolerances: the header's sizes, spacings and dt are exact; div B (rounding-level numbers) within
1e-13; the planes within 1e-13 relative L-infinity per plane (the primitives are one division
apart from the reference's).
"""
import numpy as np
import pytest

from conftest import fields, load_golden
from oracle.oracle import Oracle, rel_linf
from tests_helpers import smooth_state

pytestmark = pytest.mark.gpu

TOL = 1e-13


@pytest.fixture(scope="module")
def m():
    import torch

    assert torch.cuda.is_available()
    import magnetohydrodynamics_simulator_b200 as mod

    assert mod.device_available(), "libmhd_b200.so has no kernels for this device"
    return mod


def _planes(buf, nx, ny, ng):
    return buf[9:].reshape(7, ny + 2 * ng, nx + 2 * ng)


def _check_snapshot(got, want, nx, ny, ng):
    assert got.shape == want.shape
    assert np.array_equal(got[:7], want[:7])  # nx, ny, ng, snapshot_rate, dx, dy, dt
    assert abs(got[7] - want[7]) <= TOL and abs(got[8] - want[8]) <= TOL
    errs = [rel_linf(g, w) for g, w in zip(_planes(got, nx, ny, ng), _planes(want, nx, ny, ng))]
    assert max(errs) <= TOL, errs


def test_pack_matches_reference_file(m):
    d = load_golden("snapshot20x14_ref.npz")
    nx, ny, ng = int(d["nx"]), int(d["ny"]), int(d["ng"])
    ctx = m.Context(nx, ny, float(d["dx"]), float(d["dy"]), float(d["eta"]))
    ctx.set_state(fields(d, "state"))
    got = ctx.snapshot_pack(ng, int(d["snapshot_rate"]), float(d["dt"]))
    _check_snapshot(got, d["snapshot"], nx, ny, ng)


@pytest.mark.parametrize("nx,ny,ng", [(33, 17, 0), (33, 17, 1), (33, 17, 2), (8, 40, 3), (2, 2, 2)])
def test_pack_matches_oracle(m, nx, ny, ng):
    dx, dy = 2 * np.pi / nx, 1.5 * np.pi / ny
    ic = smooth_state(nx, ny, dx, dy, 11)
    ctx = m.Context(nx, ny, dx, dy, 1e-2)
    ctx.set_state(ic)
    ctx.step(1e-3)
    state = ctx.get_state()
    o = Oracle(nx, ny, dx, dy, 1e-2)
    o.set_state(state)
    _check_snapshot(ctx.snapshot_pack(ng, 7, 1e-3), o.snapshot(ng, 7, 1e-3), nx, ny, ng)


def test_files_written_while_stepping(m, tmp_path):
    """Snapshots written asynchronously between steps hold the state of their own step: each file
    equals the synchronous pack of a second context stepped alike (bit for bit), and reads back
    with the reference reader's slicing (scripts/display_functions.py:3-22)."""
    nx, ny, ng, dt = 96, 64, 2, 1e-3
    dx, dy = 2 * np.pi / nx, 2 * np.pi / ny
    ic = smooth_state(nx, ny, dx, dy, 5)
    a = m.Context(nx, ny, dx, dy, 5e-3)
    b = m.Context(nx, ny, dx, dy, 5e-3)
    a.set_state(ic)
    b.set_state(ic)
    paths = [str(tmp_path / f"snapshot_{k:06d}.dat") for k in range(5)]
    for p in paths:  # no synchronisation between the steps and the writes
        a.step(dt)
        a.snapshot_write(p, ng, 1, dt)
    a.snapshot_wait()
    for p in paths:
        b.step(dt)
        want = b.snapshot_pack(ng, 1, dt)
        with open(p, "rb") as f:
            raw = f.read()
        assert raw == want.tobytes()
    # the reference reader: header, then reshape(-1, nyt, nxt) and strip the ghosts
    data = np.fromfile(paths[-1], dtype=np.float64)
    nxt, nyt, g = int(data[0]) + 2 * int(data[2]), int(data[1]) + 2 * int(data[2]), int(data[2])
    planes = data[9:].reshape(-1, nyt, nxt)
    state = a.get_state()
    prim = a.primitives()
    assert np.array_equal(planes[1, g:-g, g:-g], state[3])  # E as stored
    assert np.array_equal(planes[0, g:-g, g:-g], prim["rho"])  # floored density
    for q, name in ((2, "p"), (3, "vx"), (4, "vy"), (5, "bxc"), (6, "byc")):
        assert rel_linf(planes[q, g:-g, g:-g], prim[name]) <= TOL, name


def test_unwritable_path_is_reported(m, tmp_path):
    nx = ny = 16
    ctx = m.Context(nx, ny, 2 * np.pi / nx, 2 * np.pi / ny, 1e-3)
    ctx.set_state(smooth_state(nx, ny, 2 * np.pi / nx, 2 * np.pi / ny, 3))
    ctx.snapshot_write(str(tmp_path / "no_such_dir" / "snapshot.dat"))
    with pytest.raises(m.MHDError) as e:
        ctx.snapshot_wait()
    assert e.value.status == 10  # MHD_ERR_IO
    ctx.snapshot_write(str(tmp_path / "ok.dat"))  # the context stays usable
    ctx.snapshot_wait()
    assert (tmp_path / "ok.dat").stat().st_size == ctx.snapshot_bytes(2)


def test_invalid_ghost_width(m):
    ctx = m.Context(8, 6, 0.5, 0.5, 1e-3)
    ctx.set_state(smooth_state(8, 6, 0.5, 0.5, 1))
    assert ctx.snapshot_bytes(-1) == 0 and ctx.snapshot_bytes(7) == 0
    assert ctx.snapshot_bytes(6) == 8 * (9 + 7 * 20 * 18)
    with pytest.raises(m.MHDError):
        ctx.snapshot_pack(7)
