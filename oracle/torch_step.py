"""Test infrastructure only: a PyTorch FP64 restatement of the ARS(2,2,2) IMEX step, used as the
reference adjoint (autograd) for the hand-written adjoint kernels.

It follows the CPU oracle (oracle/mhd_oracle.c) operation by operation on dense periodic planes
(index [j, i]), which in turn follows the reference solver (solvers.hpp:393-613, MUSCL.hpp,
HLL.hpp, Grid.hpp:82-136). The implicit solves use a dense direct solve of (I - alpha L), so the
gradient is exact (the reference's CG converges to machine precision on these systems); this
limits it to small grids. Floors are clamps (zero derivative where active). Nothing here is part
of the product path.
"""
from __future__ import annotations

import math

import torch

GAMMA = 5.0 / 3.0
RHO_FLOOR = 1e-8
P_FLOOR = 1e-8
G_ARS = (2.0 - math.sqrt(2.0)) / 2.0          # solvers.hpp:41
D_ARS = 1.0 - 1.0 / (2.0 * G_ARS)             # solvers.hpp:42


def at(f, di, dj):
    """f(i + di, j + dj) on the periodic grid."""
    return torch.roll(f, shifts=(-dj, -di), dims=(0, 1))


def _floor(x, fl):
    return torch.where(x < fl, torch.full_like(x, fl), x)


def primitives(U):
    """Grid.hpp:82-136 (oracle orc_primitives): rho (floored), vx, vy, p (floored), bxc, byc."""
    rho_raw, mx, my, E, bx, by = U
    bxc = (bx + at(bx, 1, 0)) / 2.0
    byc = (by + at(by, 0, 1)) / 2.0
    vx = mx / rho_raw
    vy = my / rho_raw
    rho = _floor(rho_raw, RHO_FLOOR)
    kin = 0.5 * rho * (vx * vx + vy * vy)
    mag = (bxc * bxc + byc * byc) / 2
    p = _floor((GAMMA - 1) * (E - kin - mag), P_FLOOR)
    return rho, vx, vy, p, bxc, byc


def minmod(a, b):
    """MUSCL.hpp:11-17."""
    return torch.where(a * b > 0.0, torch.where(a.abs() < b.abs(), a, b), torch.zeros_like(a))


def recon(q, dim):
    """MUSCL.hpp:26-47 along x (dim 'x') or y: (lower, upper) face values of every cell."""
    di, dj = (1, 0) if dim == "x" else (0, 1)
    s = minmod(q - at(q, -di, -dj), at(q, di, dj) - q)
    return q - 0.5 * s, q + 0.5 * s


def _safe_sqrt(x):
    pos = x > 0.0
    return torch.where(pos, torch.sqrt(torch.where(pos, x, torch.ones_like(x))), torch.zeros_like(x))


def fast_speed(rho, p, bx, by, bn):
    """HLL.hpp:107-122."""
    b2 = bx * bx + by * by
    a2 = GAMMA * p / rho
    t2 = b2 / rho
    n2 = bn * bn / rho
    s = t2 + a2
    term = s * s - 4.0 * a2 * n2
    return torch.sqrt(0.5 * (s + _safe_sqrt(term)))


def phys_flux(w, dim):
    """HLL.hpp:61-104: (rho, mx, my, E, tangential B) fluxes."""
    rho, vx, vy, p, bx, by = w
    v2 = vx * vx + vy * vy
    b2 = bx * bx + by * by
    pt = p + 0.5 * b2
    vb = vx * bx + vy * by
    E = p / (GAMMA - 1.0) + 0.5 * (rho * v2 + b2)
    if dim == "x":
        return (rho * vx, rho * vx * vx + pt - bx * bx, rho * vx * vy - bx * by,
                (E + pt) * vx - bx * vb, vx * by - vy * bx)
    return (rho * vy, rho * vx * vy - bx * by, rho * vy * vy + pt - by * by,
            (E + pt) * vy - by * vb, vy * bx - vx * by)


def conserved(w, dim):
    """HLL.hpp:31-47."""
    rho, vx, vy, p, bx, by = w
    v2 = vx * vx + vy * vy
    b2 = bx * bx + by * by
    return (rho, rho * vx, rho * vy, p / (GAMMA - 1.0) + 0.5 * rho * v2 + 0.5 * b2,
            by if dim == "x" else bx)


def hll(Lw, Rw, dim):
    """HLL.hpp:126-218."""
    FL, FR = phys_flux(Lw, dim), phys_flux(Rw, dim)
    if dim == "x":
        cL = fast_speed(Lw[0], Lw[3], Lw[4], Lw[5], Lw[4])
        cR = fast_speed(Rw[0], Rw[3], Rw[4], Rw[5], Rw[4])
        vL, vR = Lw[1], Rw[1]
    else:
        cL = fast_speed(Lw[0], Lw[3], Lw[4], Lw[5], Lw[5])
        cR = fast_speed(Rw[0], Rw[3], Rw[4], Rw[5], Rw[5])
        vL, vR = Lw[2], Rw[2]
    a, b = vL - cL, vR - cR
    sL = torch.where(b < a, b, a)           # std::min
    a, b = vL + cL, vR + cR
    sR = torch.where(a < b, b, a)           # std::max
    UL, UR = conserved(Lw, dim), conserved(Rw, dim)
    den = torch.where(sR - sL != 0.0, sR - sL, torch.ones_like(sL))
    inv = 1.0 / den
    out = []
    for fl, fr, ul, ur in zip(FL, FR, UL, UR):
        avg = (sR * fl - sL * fr + sL * sR * (ur - ul)) * inv
        out.append(torch.where(sL >= 0, fl, torch.where(sR <= 0, fr, avg)))
    return out


def ct_average(v, mode):
    """solvers.hpp:326,333 (mode 0: the int-truncating abs the reference compiles to)."""
    if mode == 1:
        return v.abs() < 1e-12
    return ~((v.abs() >= 1.0) & (v.abs() < 2147483648.0))


def explicit_rhs(U, dx, dy, ct_mode=0):
    """solvers.hpp:393-402 (oracle orc_explicit_rhs): the six rates."""
    rho, vx, vy, p, bxc, byc = primitives(U)
    bxf, byf = U[4], U[5]
    # x faces: L = upper extrapolation of cell i, R = lower extrapolation of cell i+1, Bn = bxf(i+1)
    lo = [recon(q, "x") for q in (rho, vx, vy, p, byc)]
    Lx = [l[1] for l in lo]
    Rx = [at(l[0], 1, 0) for l in lo]
    bn = at(bxf, 1, 0)
    Lw = (Lx[0], Lx[1], Lx[2], Lx[3], bn, Lx[4])
    Rw = (Rx[0], Rx[1], Rx[2], Rx[3], bn, Rx[4])
    Fx = hll(Lw, Rw, "x")
    # y faces: D = upper extrapolation of cell j, U = lower extrapolation of cell j+1, Bn = byf(j+1)
    lo = [recon(q, "y") for q in (rho, vx, vy, p, bxc)]
    Dy = [l[1] for l in lo]
    Uy = [at(l[0], 0, 1) for l in lo]
    bn = at(byf, 0, 1)
    Dw = (Dy[0], Dy[1], Dy[2], Dy[3], Dy[4], bn)
    Uw = (Uy[0], Uy[1], Uy[2], Uy[3], Uy[4], bn)
    Fy = hll(Dw, Uw, "y")
    # corner Ez (solvers.hpp:294-346)
    eN = -at(Fx[4], -1, 0)
    eS = -at(Fx[4], -1, -1)
    eE = at(Fy[4], 0, -1)
    eW = at(Fy[4], -1, -1)
    vxc = 0.25 * (vx + at(vx, -1, 0) + at(vx, 0, -1) + at(vx, -1, -1))
    vyc = 0.25 * (vy + at(vy, -1, 0) + at(vy, 0, -1) + at(vy, -1, -1))
    ezy = torch.where(ct_average(vyc, ct_mode), 0.5 * (eS + eN), torch.where(vyc > 0.0, eS, eN))
    ezx = torch.where(ct_average(vxc, ct_mode), 0.5 * (eE + eW), torch.where(vxc > 0.0, eW, eE))
    ez = 0.5 * (ezx + ezy)
    rates = []
    for q in range(4):
        rates.append(-((Fx[q] - at(Fx[q], -1, 0)) / dx + (Fy[q] - at(Fy[q], 0, -1)) / dy))
    rates.append(-(at(ez, 0, 1) - ez) / dy)
    rates.append((at(ez, 1, 0) - ez) / dx)
    return rates


def corner_current(bx, by, dx, dy):
    """solvers.hpp:450-461 without eta: J_z at the bottom-left corner of every cell."""
    return (by - at(by, -1, 0)) / dx - (bx - at(bx, 0, -1)) / dy


def curl_rate(E, dx, dy):
    """solvers.hpp:478-486: (rate of bxf, rate of byf) = -curl of the corner field."""
    return -(at(E, 0, 1) - E) / dy, (at(E, 1, 0) - E) / dx


def laplacian_matrix(nx, ny, dx, dy, dtype=torch.float64):
    """The corner Laplacian L of solvers.hpp:404-443 (periodic 5-point) as a dense matrix."""
    n = nx * ny
    L = torch.zeros((n, n), dtype=dtype)
    for j in range(ny):
        for i in range(nx):
            r = j * nx + i
            L[r, r] += -2.0 / dx**2 - 2.0 / dy**2
            L[r, j * nx + (i - 1) % nx] += 1.0 / dx**2
            L[r, j * nx + (i + 1) % nx] += 1.0 / dx**2
            L[r, ((j - 1) % ny) * nx + i] += 1.0 / dy**2
            L[r, ((j + 1) % ny) * nx + i] += 1.0 / dy**2
    return L


def resistive_rate(bx, by, eta, alpha, Lmat, dx, dy):
    """solvers.hpp:445-489: implicit (alpha given) or explicit (alpha None) rate of the face B."""
    rhs = eta * corner_current(bx, by, dx, dy)
    if alpha is None:
        E = rhs
    else:
        n = rhs.numel()
        M = torch.eye(n, dtype=rhs.dtype, device=rhs.device) - alpha * Lmat
        E = torch.linalg.solve(M, rhs.reshape(-1)).reshape(rhs.shape)
    return curl_rate(E, dx, dy)


def imex_step(U, dt, eta, dx, dy, Lmat, ct_mode=0):
    """solvers.hpp:491-613 (oracle orc_imex_step) with alpha = dt*eta*g (the driver's matrix for a
    fixed dt). U: list of six (ny, nx) tensors; eta may be a tensor (for its gradient)."""
    alpha = (dt * eta) * G_ARS
    ini = list(U)
    f1 = explicit_rhs(U, dx, dy, ct_mode)
    s = list(U)
    s[0] = _floor(s[0], RHO_FLOOR)
    c1 = dt * G_ARS
    u1 = [ini[k] + f1[k] * c1 for k in range(6)]
    u1[0] = _floor(u1[0], RHO_FLOOR)
    sx, sy = resistive_rate(u1[4], u1[5], eta, alpha, Lmat, dx, dy)
    diag = dt * G_ARS
    u1[4] = u1[4] + sx * diag
    u1[5] = u1[5] + sy * diag
    f2 = explicit_rhs(u1, dx, dy, ct_mode)
    gx, gy = resistive_rate(u1[4], u1[5], eta, None, Lmat, dx, dy)
    c2, c3, ci3 = dt * D_ARS, dt * (1.0 - D_ARS), dt * (1.0 - G_ARS)
    u2 = [ini[k] + f1[k] * c2 + f2[k] * c3 for k in range(6)]
    u2[4] = u2[4] + gx * ci3
    u2[5] = u2[5] + gy * ci3
    u2[0] = _floor(u2[0], RHO_FLOOR)
    sx, sy = resistive_rate(u2[4], u2[5], eta, alpha, Lmat, dx, dy)
    u2[4] = u2[4] + sx * diag
    u2[5] = u2[5] + sy * diag
    g3x, g3y = resistive_rate(u2[4], u2[5], eta, None, Lmat, dx, dy)
    fc1, fc2, gc2, gc3 = dt * D_ARS, dt * (1.0 - D_ARS), dt * (1.0 - G_ARS), dt * G_ARS
    out = [s[k] + f1[k] * fc1 + f2[k] * fc2 for k in range(6)]
    out[4] = out[4] + gx * gc2 + g3x * gc3
    out[5] = out[5] + gy * gc2 + g3y * gc3
    out[0] = _floor(out[0], RHO_FLOOR)
    return out


def state_from_potential(az, rho, vx, vy, p, dx, dy):
    """Face B = curl Az from corner values (benchmarks.hpp:58-59) and the conserved state with E
    from the cell-averaged face B. az: (ny+1, nx+1) corner values (periodic: last row/column
    repeat the first)."""
    bx = (az[1:, :-1] - az[:-1, :-1]) / dy
    by = -(az[:-1, 1:] - az[:-1, :-1]) / dx
    bxc = 0.5 * (bx + at(bx, 1, 0))
    byc = 0.5 * (by + at(by, 0, 1))
    E = p / (GAMMA - 1.0) + 0.5 * rho * (vx * vx + vy * vy) + 0.5 * (bxc * bxc + byc * byc)
    return [rho, rho * vx, rho * vy, E, bx, by]
