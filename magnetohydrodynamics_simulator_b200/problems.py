"""Initial conditions of the benchmark configurations, built on the host in numpy.

Orszag-Tang and the decaying magnetic sine wave follow the reference's initial-condition
functions (include/benchmarks.hpp:15-76 and :352-417): face B from a vector potential sampled at
cell corners, total energy from the face values. The other five (Alfven wave, Gaussian density
pulse, acoustic wave, sausage and kink pinches, benchmarks.hpp:78-350) set face B from cell-centre
formulas, as the reference does. The mixed-size batch generator builds the
synthetic ensemble of independent periodic runs (smoothed random density, Fourier-mode velocity
and vector potential). Fields are returned as dense (ny, nx) float64 arrays in the order rho, mx,
my, E, bxf, byf.
"""
from __future__ import annotations

import numpy as np

GAMMA_GAS = 5.0 / 3.0
PI_REF = 3.14159265359  # the reference driver's pi literal (src/integrator_main.cpp:36)


def grid_spacing(n: int) -> float:
    """dx = 2*pi/n with the reference driver's pi (integrator_main.cpp:37-38)."""
    return 2 * PI_REF / n


def _from_potential(az, rho0, p0, vx, vy, dx, dy):
    bxf = (az[1:, :-1] - az[:-1, :-1]) / dy
    byf = -(az[:-1, 1:] - az[:-1, :-1]) / dx
    E = p0 / (GAMMA_GAS - 1.0) + 0.5 * rho0 * (vx * vx + vy * vy) + 0.5 * (bxf * bxf + byf * byf)
    rho = np.full_like(vx, rho0)
    return [np.ascontiguousarray(a) for a in (rho, rho0 * vx, rho0 * vy, E, bxf, byf)]


def orszag_tang(nx: int, ny: int, dx: float, dy: float):
    """Orszag-Tang vortex: rho = 25/9, p = 5/3, v = (-sin y, sin x), Az = 0.5 cos 2x + cos y."""
    xc = np.arange(nx + 1) * dx
    yc = np.arange(ny + 1) * dy
    az = 0.5 * np.cos(2 * xc)[None, :] + np.cos(yc)[:, None]
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dy
    vx = np.broadcast_to(-np.sin(y)[:, None], (ny, nx)).copy()
    vy = np.broadcast_to(np.sin(x)[None, :], (ny, nx)).copy()
    return _from_potential(az, 25.0 / 9.0, 5.0 / 3.0, vx, vy, dx, dy)


def sine_wave(nx: int, ny: int, dx: float, dy: float, az_amp: float, kx: float, ky: float,
              use_sin: bool = True):
    """Decaying magnetic sine wave: rho = p = 1, v = 0, Az = az_amp * f(kx x) sin(ky y)."""
    xc = np.arange(nx + 1) * dx
    yc = np.arange(ny + 1) * dy
    fx = np.sin(kx * xc) if use_sin else np.cos(kx * xc)
    az = az_amp * fx[None, :] * np.sin(ky * yc)[:, None]
    z = np.zeros((ny, nx))
    return _from_potential(az, 1.0, 1.0, z, z, dx, dy)


def sine_wave_config(n: int, b0: float = 1e-3, k: float = 1.0):
    """The configured decaying wave: Az = (B0/k) sin(kx x) sin(ky y), kx = ky = k on [0, 2pi)^2."""
    dx = grid_spacing(n)
    return sine_wave(n, n, dx, dx, b0 / k, k, k, use_sin=True), dx


# ------------------------------------------------------------------ benchmarks.hpp:78-350
# The reference's other five initial conditions set every field at cell centres of the padded
# grid, face B included (each has B_x constant and B_y a function of x only, so div B = 0), and
# convert with ConservedState::fromPrimitive (HLL.hpp:31-47). Only the physical cells are returned
# (the driver's ghost fill overwrites the rest, integrator_main.cpp:52). The reference's pi literal
# and its sampling positions are kept, quirks included.


def _centres(nx, ny, dx, dy, offset=0.5):
    x = (np.arange(nx) + offset) * dx
    y = (np.arange(ny) + offset) * dy
    return np.meshgrid(x, y)


def _conserved(rho, vx, vy, p, bx, by):
    """HLL.hpp:31-47 fromPrimitive (bx, by go to the face planes unchanged)."""
    rho, vx, vy, p, bx, by = np.broadcast_arrays(rho, vx, vy, p, bx, by)
    E = p / (GAMMA_GAS - 1.0) + 0.5 * rho * (vx * vx + vy * vy) + 0.5 * (bx * bx + by * by)
    return [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, rho * vx, rho * vy, E, bx, by)]


def alfven_wave(nx: int, ny: int, dx: float, dy: float):
    """benchmarks.hpp:78-125: B_x = 1, B_y = 1e-3 sin(kx x), v_y = -B_y/sqrt(rho), rho = p = 1."""
    X, _ = _centres(nx, ny, dx, dy)
    kx = 2.0 * PI_REF / (nx * dx)
    by = 1e-3 * np.sin(kx * X)
    vy = -by / np.sqrt(1.0)
    return _conserved(1.0, 0.0, vy, 1.0, 1.0, by)


def gaussian_pulse(nx: int, ny: int, dx: float, dy: float):
    """benchmarks.hpp:127-172: rho = 1 + exp(-5 r^2 / 4) around the centre, v = (1, 1), p = 1,
    B = 0. The centre's y uses nx (y_mid = 0.5 nx dy, :140), as the reference writes it."""
    X, Y = _centres(nx, ny, dx, dy)
    x_mid, y_mid = 0.5 * nx * dx, 0.5 * nx * dy
    d2 = (X - x_mid) * (X - x_mid) + (Y - y_mid) * (Y - y_mid)
    rho = 1.0 + np.exp(-5 * d2 / (2.0 * 2.0))
    return _conserved(rho, 1.0, 1.0, 1.0, 0.0, 0.0)


def acoustic_wave(nx: int, ny: int, dx: float, dy: float):
    """benchmarks.hpp:174-231: a right-moving sound wave of amplitude 1e-4 and wavenumber 4 pi / L
    sampled at cell corners (x = i dx, :210), p0 = 1/gamma, B = 0."""
    X, _ = _centres(nx, ny, dx, dy, offset=0.0)
    p_bg = 1.0 / GAMMA_GAS
    c = np.sqrt(GAMMA_GAS * p_bg / 1.0)
    s = 1e-4 * np.sin(4 * PI_REF * X / (dx * nx))
    return _conserved(1.0 + s + 0.0, (c / 1.0) * s, (c / 1.0) * 0.0, p_bg + (c * c) * (s + 0.0), 0.0, 0.0)


def _channel_centre(nx, dx, ng=2):
    # x_mid = 0.5 * nxt * dx (benchmarks.hpp:252, :305): half the PADDED width, i.e. ng cells right
    # of the physical centre
    return 0.5 * (nx + 2 * ng) * dx


def sausage(nx: int, ny: int, dx: float, dy: float, ng: int = 2):
    """benchmarks.hpp:233-287: low-beta pinch (B_y = 5 (r/0.2) exp(-r^2/0.04), p = 0.1 exp(.) +
    0.1, rho = exp(.) + 0.1) with an m = 0 modulation 1 - 0.15 cos(2 pi y / H) of the channel."""
    X, Y = _centres(nx, ny, dx, dy)
    r = X - _channel_centre(nx, dx, ng)
    H = ny * dy
    pert = 1.0 - 0.15 * np.cos((2.0 * PI_REF / H) * Y)
    rho = np.maximum(1.0 * np.exp(-(r * r) / (0.04 * pert)) + 0.1, 1e-4)
    p = np.maximum(0.1 * np.exp(-(r * r) / (0.04 * pert)) + 0.1, 1e-4)
    by = 5.0 * (r / np.sqrt(0.04)) * np.exp(-(r * r) / 0.04)
    return _conserved(rho, 0.0, 0.0, p, 0.0, by)


def kink(nx: int, ny: int, dx: float, dy: float, ng: int = 2):
    """benchmarks.hpp:289-350: a current channel B_y = exp(-r^2/0.04), rho = p = exp(.) + 0.1,
    seeded by v_x = 0.05 sin(2 pi y) exp(-r^2/0.04)."""
    X, Y = _centres(nx, ny, dx, dy)
    r = X - _channel_centre(nx, dx, ng)
    env = np.exp(-(r * r) / 0.04)
    vx = 0.05 * np.sin((2.0 * PI_REF) * Y) * env
    return _conserved(1.0 * env + 0.1, vx, 0.0, 1.0 * env + 0.1, 0.0, 1.0 * env)


FIXTURES = {"alfven_wave": alfven_wave, "gaussian_pulse": gaussian_pulse,
            "acoustic_wave": acoustic_wave, "sausage": sausage, "kink": kink}


def _fourier_modes(rng, X, Y, Lx, Ly, n_modes, amp_lo, amp_hi, kmax=4):
    f = np.zeros_like(X)
    for _ in range(n_modes):
        while True:
            kx, ky = rng.integers(-kmax, kmax + 1, size=2)
            if (kx, ky) != (0, 0) and kx * kx + ky * ky <= kmax * kmax:
                break
        a = rng.uniform(amp_lo, amp_hi)
        ph = rng.uniform(0, 2 * np.pi)
        f += a * np.sin(2 * np.pi * (kx * X / Lx + ky * Y / Ly) + ph)
    return f


def _smooth_periodic(rng, nx, ny, width_cells):
    """N(0,1) noise smoothed by a periodic Gaussian (FFT), rescaled to unit std."""
    noise = rng.standard_normal((ny, nx))
    kx = np.fft.fftfreq(nx)[None, :]
    ky = np.fft.fftfreq(ny)[:, None]
    filt = np.exp(-0.5 * (2 * np.pi * width_cells) ** 2 * (kx * kx + ky * ky))
    s = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    sd = s.std()
    return s / sd if sd > 0 else s


def random_instance(n: int, seed: int, v_modes: int = 8, az_modes: int = 8, rho_floor: float = 0.2):
    """One member of the mixed-size batch: rho = 1 + 0.2 * smoothed N(0,1) (clamped at rho_floor),
    p = 1, v and Az sums of Fourier modes with |k| <= 4 and per-mode amplitudes in [0.1, 1] (the
    sums are not normalised: |v| reaches ~4-5 and |B| ~5-7, supersonic and low-beta)."""
    rng = np.random.default_rng(seed)
    dx = grid_spacing(n)
    L = n * dx
    x = (np.arange(n) + 0.5) * dx
    X, Y = np.meshgrid(x, x)
    xc = np.arange(n + 1) * dx
    XC, YC = np.meshgrid(xc, xc)
    rho = np.maximum(1.0 + 0.2 * _smooth_periodic(rng, n, n, width_cells=n / 32), rho_floor)
    vx = _fourier_modes(rng, X, Y, L, L, v_modes, 0.1, 1.0)
    vy = _fourier_modes(rng, X, Y, L, L, v_modes, 0.1, 1.0)
    az = _fourier_modes(rng, XC, YC, L, L, az_modes, 0.1, 1.0)
    bxf = (az[1:, :-1] - az[:-1, :-1]) / dx
    byf = -(az[:-1, 1:] - az[:-1, :-1]) / dx
    bxc = 0.5 * (bxf + np.roll(bxf, -1, axis=1))
    byc = 0.5 * (byf + np.roll(byf, -1, axis=0))
    p = 1.0
    E = p / (GAMMA_GAS - 1.0) + 0.5 * rho * (vx * vx + vy * vy) + 0.5 * (bxc * bxc + byc * byc)
    fields = [np.ascontiguousarray(a) for a in (rho, rho * vx, rho * vy, E, bxf, byf)]
    return fields, dx


def mixed_batch(count: int = 64, seed: int = 2024, sizes=(256, 384, 512, 768, 1024)):
    """Seeded sizes and resistivities of the mixed-size batch: eta log-uniform in [1e-4, 1e-2]."""
    rng = np.random.default_rng(seed)
    ns = rng.choice(np.array(sizes), size=count)
    etas = np.exp(rng.uniform(np.log(1e-4), np.log(1e-2), size=count))
    seeds = rng.integers(0, 2**31 - 1, size=count)
    return [(int(n), float(e), int(s)) for n, e, s in zip(ns, etas, seeds)]
