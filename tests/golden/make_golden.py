"""Generate the golden fixtures in this folder from the reference solver's own code.

Run here (where the reference sources exist), never on the GPU box:

    make -C oracle ref && python tests/golden/make_golden.py

Every fixture is produced by ``oracle/_ref/libmhdref.so`` -- the reference's include/*.hpp compiled
unmodified (with the project-written Eigen subset), driven by oracle/ref_harness.cpp. Inputs that
the reference has no initial-condition function for (random smooth states, the configured
decaying-wave amplitude) are built in numpy with a fixed seed and loaded into the reference's Grid
through ``ref_set_state``; the stored input is exactly what the reference stepped.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import PI_REF, Oracle, Reference, build, default_alpha  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def smooth_random_state(nx, ny, dx, dy, seed, n_modes=6, v_amp=0.3, az_amp=0.2):
    """A smooth periodic state: rho, p positive; B = curl Az on faces (divergence-free)."""
    rng = np.random.default_rng(seed)
    Lx, Ly = nx * dx, ny * dy
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(x, y)
    xc = np.arange(nx + 1) * dx
    yc = np.arange(ny + 1) * dy
    XC, YC = np.meshgrid(xc, yc)

    def modes(XX, YY, amp):
        f = np.zeros_like(XX)
        for _ in range(n_modes):
            kx, ky = rng.integers(-3, 4, size=2)
            ph = rng.uniform(0, 2 * np.pi)
            a = rng.uniform(0.3, 1.0) * amp
            f += a * np.sin(2 * np.pi * (kx * XX / Lx + ky * YY / Ly) + ph)
        return f

    rho = 1.0 + 0.5 * np.tanh(modes(X, Y, 0.5))
    p = 1.0 + 0.3 * np.tanh(modes(X, Y, 0.5))
    vx = modes(X, Y, v_amp)
    vy = modes(X, Y, v_amp)
    az = modes(XC, YC, az_amp)
    bxf = (az[1:, :-1] - az[:-1, :-1]) / dy
    byf = -(az[:-1, 1:] - az[:-1, :-1]) / dx
    # E from the cell-averaged B so the stored pressure is p
    bxc = 0.5 * (bxf + np.roll(bxf, -1, axis=1))
    byc = 0.5 * (byf + np.roll(byf, -1, axis=0))
    E = p / (5.0 / 3.0 - 1.0) + 0.5 * rho * (vx**2 + vy**2) + 0.5 * (bxc**2 + byc**2)
    return [np.ascontiguousarray(a) for a in (rho, rho * vx, rho * vy, E, bxf, byf)]


def pack(prefix, fields):
    return {f"{prefix}_{n}": f for n, f in zip(("rho", "mx", "my", "E", "bxf", "byf"), fields)}


def ot(n, eta, steps, with_inputs=True):
    dx = 2 * PI_REF / n
    ref = Reference(n, n, dx, dx, eta)
    ref.init_orszag_tang()
    ic = ref.get_state()
    f1 = ref.explicit_rhs()
    dts, prods = ref.run(steps)
    out = dict(nx=n, ny=n, dx=dx, dy=dx, eta=eta, steps=steps, dts=dts, cg_products=prods)
    if with_inputs:  # the initial condition is also rebuilt by the oracle's own IC function
        out.update(pack("ic", ic))
        out.update(pack("f1", f1))
    out.update(pack("final", ref.get_state()))
    out["divb"] = np.array(ref.divb())
    return out


def main():
    build(with_reference=True)

    # 1. Orszag-Tang 32^2, eta = 1e-3, reference driver loop (dynamic CFL), 20 steps
    np.savez(os.path.join(OUT, "ot32_ref.npz"), **ot(32, 1e-3, 20))

    # 2. Orszag-Tang 128^2, eta = 1e-3, 200 steps (the CPU-runnable configuration)
    np.savez(os.path.join(OUT, "ot128_ref.npz"), **ot(128, 1e-3, 200, with_inputs=False))

    # 3. Decaying magnetic sine wave, configured variant: Az = 1e-3 sin x sin y, eta = 10,
    #    fixed dt = 1e-4, 64^2, 20 steps (CG-dominated: tens of iterations per solve)
    n = 64
    dx = 2 * PI_REF / n
    orc = Oracle(n, n, dx, dx, 10.0)
    orc.init_sine_wave(az_amp=1e-3, kx=1.0, ky=1.0, use_sin=True)
    ic = orc.get_state()
    ref = Reference(n, n, dx, dx, 10.0)
    ref.set_state(ic)
    dts, prods = ref.run(20, dt_fixed=1e-4)
    out = dict(nx=n, ny=n, dx=dx, dy=dx, eta=10.0, steps=20, dts=dts, cg_products=prods)
    out.update(pack("ic", ref_state_after_set(ic, n, dx, 10.0)))
    out.update(pack("final", ref.get_state()))
    out["divb"] = np.array(ref.divb())
    np.savez(os.path.join(OUT, "dsw64_ref.npz"), **out)

    # 4. The reference's own decaying-wave initial condition (benchmarks.hpp:352-417), 32^2
    n = 32
    dx = 2 * PI_REF / n
    ref = Reference(n, n, dx, dx, 10.0)
    ref.init_dsw()
    ic = ref.get_state()
    dts, prods = ref.run(5, dt_fixed=1e-4)
    out = dict(nx=n, ny=n, dx=dx, dy=dx, eta=10.0, steps=5, dts=dts, cg_products=prods)
    out.update(pack("ic", ic))
    out.update(pack("final", ref.get_state()))
    np.savez(os.path.join(OUT, "dswref32_ref.npz"), **out)

    # 5. Random smooth state on a non-square grid with dx != dy: f1, one implicit rate, 3 steps
    nx, ny = 40, 24
    dx, dy = 2 * PI_REF / nx, 1.5 * PI_REF / ny
    eta = 2e-2
    ic = smooth_random_state(nx, ny, dx, dy, seed=1234)
    ref = Reference(nx, ny, dx, dy, eta)
    ref.set_state(ic)
    f1 = ref.explicit_rhs()
    dt = 0.5 * ref.cfl_dt()
    ref.set_alpha(default_alpha(dt, eta))
    sbx, sby, jz = ref.implicit_rate()
    dts, prods = ref.run(3, dt_fixed=dt)
    out = dict(nx=nx, ny=ny, dx=dx, dy=dy, eta=eta, steps=3, dts=dts, cg_products=prods,
               implicit_alpha=default_alpha(dt, eta), implicit_bx=sbx, implicit_by=sby, implicit_rhs=jz)
    out.update(pack("ic", ic))
    out.update(pack("f1", f1))
    out.update(pack("final", ref.get_state()))
    np.savez(os.path.join(OUT, "random40x24_ref.npz"), **out)

    # 6. Upwind branch of the corner field: velocities above 1 so the (int-truncated) corner
    #    test selects upwinding; 32x32, eta = 0 (the implicit solves return at once)
    nx = ny = 32
    dx = dy = 2 * PI_REF / nx
    ic = smooth_random_state(nx, ny, dx, dy, seed=77, v_amp=1.6, az_amp=0.3)
    ref = Reference(nx, ny, dx, dy, 0.0)
    ref.set_state(ic)
    f1 = ref.explicit_rhs()
    dts, prods = ref.run(5)
    out = dict(nx=nx, ny=ny, dx=dx, dy=dy, eta=0.0, steps=5, dts=dts, cg_products=prods)
    out.update(pack("ic", ic))
    out.update(pack("f1", f1))
    out.update(pack("final", ref.get_state()))
    np.savez(os.path.join(OUT, "upwind32_ref.npz"), **out)

    # 7. Snapshot file (diagnostics.hpp:90-131) of a random smooth state on a 20x14 grid with
    #    dx != dy after 2 reference steps: the exact bytes the reference writes, ng = 2
    nx, ny = 20, 14
    dx, dy = 2 * PI_REF / nx, 1.25 * PI_REF / ny
    eta = 1e-2
    ref = Reference(nx, ny, dx, dy, eta)
    ref.set_state(smooth_random_state(nx, ny, dx, dy, seed=4321))
    dts, _ = ref.run(2)
    with tempfile.TemporaryDirectory() as tmp:
        raw = ref.write_snapshot(tmp, 3, 5, float(dts[-1]))
    out = dict(nx=nx, ny=ny, dx=dx, dy=dy, eta=eta, ng=2, snapshot_rate=5, frame_index=3,
               dt=float(dts[-1]), snapshot=np.frombuffer(raw, dtype=np.float64))
    out.update(pack("state", ref.get_state()))
    np.savez(os.path.join(OUT, "snapshot20x14_ref.npz"), **out)

    # 8. The reference's five other initial conditions (benchmarks.hpp:78-350) on a 32x24 grid with
    #    dx != dy, and 5 steps of the reference driver loop from each (dynamic CFL, eta = 5e-3)
    nx, ny = 32, 24
    dx, dy = 2 * PI_REF / nx, 1.5 * PI_REF / ny
    eta = 5e-3
    out = dict(nx=nx, ny=ny, dx=dx, dy=dy, eta=eta, steps=5, names=np.array(Reference.FIXTURES))
    for name in Reference.FIXTURES:
        ref = Reference(nx, ny, dx, dy, eta)
        ref.init_fixture(name)
        out.update(pack(f"{name}_ic", ref.get_state()))
        dts, prods = ref.run(5)
        out[f"{name}_dts"] = dts
        out[f"{name}_cg_products"] = prods
        out.update(pack(f"{name}_final", ref.get_state()))
    np.savez(os.path.join(OUT, "fixtures32x24_ref.npz"), **out)

    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))


def ref_state_after_set(ic, n, dx, eta):
    ref = Reference(n, n, dx, dx, eta)
    ref.set_state(ic)
    return ref.get_state()


if __name__ == "__main__":
    main()
