"""Test infrastructure only: a CPU stand-in for one subdomain of the domain decomposition, with the
same methods as magnetohydrodynamics_simulator_b200.decomposed.GpuSubdomain, so that the
decomposition driver (partition, ring exchanges, ordered reductions, the distributed CG) can be
tested on the CPU, over gloo ranks, against the single-domain C oracle.

The subdomain keeps extended planes of (nx + 2H) x (ny + 2H) cells like the GPU one and computes
the stages in the GPU kernels' split (U1* = U + dt g f1, accumulator = floor(U) + dt d f1, then
+ dt (1-d) f2 + dt (1-g) g2 on the faces; B^{n+1} = U2*_B + dt g g3) with the oracle's explicit
rate and explicit resistive rate (oracle/mhd_oracle.c) applied to the extended planes as a periodic
grid: the interior is exact when the rings hold the neighbours' values (orc_explicit_rhs follows
solvers.hpp:393-402, orc_resistive_rate solvers.hpp:445-489 with solve_implicitly = false).
"""
from __future__ import annotations

import ctypes

import numpy as np

from oracle.oracle import Oracle, _ptr

H = 4
WEST, EAST, SOUTH, NORTH = 0, 1, 2, 3
RHO_FLOOR = 1e-8
GAMMA = 5.0 / 3.0


class OracleSubdomain:
    def __init__(self, nx, ny, dx, dy, eta):
        self.nx, self.ny, self.dx, self.dy, self.eta = nx, ny, dx, dy, eta
        self.nxe, self.nye = nx + 2 * H, ny + 2 * H
        self.orc = Oracle(self.nxe, self.nye, dx, dy, eta)
        z = lambda: np.zeros((self.nye, self.nxe))  # noqa: E731
        self.S = [z() for _ in range(6)]
        self.T = [z() for _ in range(6)]
        self.A = [z() for _ in range(6)]
        self.x, self.r, self.p, self.q, self.zv = z(), z(), z(), z(), z()
        self.g = (2.0 - np.sqrt(2.0)) / 2.0
        self.d = 1.0 - 1.0 / (2.0 * self.g)
        self.I = (slice(H, H + ny), slice(H, H + nx))

    # -- state and rings
    def set_state(self, fields):
        for k in range(6):
            self.S[k][self.I] = fields[k]

    def get_state(self):
        return [self.S[k][self.I].copy() for k in range(6)]

    def _planes(self, set_):
        return {0: self.S, 1: self.T, 2: [self.A[4], self.A[5]], 3: [self.x], 4: [self.p]}[set_]

    def _rect(self, side, width, send):
        nx, ny = self.nx, self.ny
        if side == WEST:
            return slice(H, H + ny), (slice(H, H + width) if send else slice(H - width, H))
        if side == EAST:
            return slice(H, H + ny), (slice(H + nx - width, H + nx) if send else slice(H + nx, H + nx + width))
        if side == SOUTH:
            return (slice(H, H + width) if send else slice(H - width, H)), slice(0, self.nxe)
        return (slice(H + ny - width, H + ny) if send else slice(H + ny, H + ny + width)), slice(0, self.nxe)

    def pack(self, set_, side, width):
        rs, cs = self._rect(side, width, True)
        return np.concatenate([pl[rs, cs].ravel() for pl in self._planes(set_)])

    def unpack(self, set_, side, width, buf):
        rs, cs = self._rect(side, width, False)
        planes = self._planes(set_)
        per = buf.size // len(planes)
        for k, pl in enumerate(planes):
            pl[rs, cs] = np.asarray(buf[k * per:(k + 1) * per]).reshape(pl[rs, cs].shape)

    def synchronize(self):
        pass

    # -- diagnostics
    def cfl_speed(self):
        u = [f for f in self.S]
        I = self.I
        bxc = (u[4][I] + np.roll(u[4], -1, axis=1)[I]) / 2.0
        byc = (u[5][I] + np.roll(u[5], -1, axis=0)[I]) / 2.0
        rho = u[0][I]
        vx, vy = u[1][I] * (1.0 / rho), u[2][I] * (1.0 / rho)
        rho_f = np.where(rho < RHO_FLOOR, RHO_FLOOR, rho)
        kin = 0.5 * rho_f * (vx * vx + vy * vy)
        mag = (bxc * bxc + byc * byc) / 2
        p = (GAMMA - 1) * (u[3][I] - kin - mag)
        p = np.where(p < 1e-8, 1e-8, p)
        r = np.maximum(rho_f, 1e-8)
        pr = np.maximum(p, 1e-8)
        ir = 1.0 / r
        sp = np.sqrt(GAMMA * pr * ir + (bxc * bxc + byc * byc) * ir) + np.sqrt(vx * vx + vy * vy)
        bad = not all(np.all(np.isfinite(f[I])) for f in u)
        return float(np.max(sp)), bad

    def divb_sums(self):
        I = self.I
        d = (np.roll(self.S[4], -1, axis=1)[I] - self.S[4][I]) / self.dx + \
            (np.roll(self.S[5], -1, axis=0)[I] - self.S[5][I]) / self.dy
        return [float(np.sum(d * d)), float(np.max(np.abs(d)))]

    # -- step
    def set_step(self, dt, alpha):
        self.dt, self.alpha = dt, alpha
        self.c_g, self.c_d = dt * self.g, dt * self.d
        self.c_1md, self.c_1mg = dt * (1.0 - self.d), dt * (1.0 - self.g)
        self.cx = alpha / (self.dx * self.dx)
        self.cy = alpha / (self.dy * self.dy)
        self.diag = 1 + 2 * (self.cx + self.cy)
        self.invdiag = 1.0 if self.diag == 0.0 else 1.0 / self.diag

    def _rhs(self, planes):
        self.orc.set_state(planes)
        return self.orc.explicit_rhs()

    def _resistive(self, bx, by):
        """Explicit resistive rate -curl(eta J_z(B)) on the extended planes (periodic)."""
        gx, gy = np.zeros_like(bx), np.zeros_like(by)
        bx, by = np.ascontiguousarray(bx), np.ascontiguousarray(by)
        self.orc.lib.orc_resistive_rate(ctypes.byref(self.orc.p), _ptr(bx), _ptr(by), -1.0, _ptr(gx), _ptr(gy))
        return gx, gy

    def _rate(self, e):
        """Face rate of a corner field: (-(E(i,j+1) - E(i,j))/dy, (E(i+1,j) - E(i,j))/dx)."""
        return -(np.roll(e, -1, axis=0) - e) / self.dy, (np.roll(e, -1, axis=1) - e) / self.dx

    def stage(self, k):
        if k == 1:
            f1 = self._rhs(self.S)
            for q in range(6):
                self.T[q] = self.S[q] + f1[q] * self.c_g
                u = np.where(self.S[0] < RHO_FLOOR, RHO_FLOOR, self.S[0]) if q == 0 else self.S[q]
                self.A[q] = u + f1[q] * self.c_d
        else:
            rx, ry = self._rate(self.x)
            b1x = self.T[4] + rx * self.c_g
            b1y = self.T[5] + ry * self.c_g
            u1 = [np.where(self.T[0] < RHO_FLOOR, RHO_FLOOR, self.T[0]), self.T[1], self.T[2], self.T[3], b1x, b1y]
            f2 = self._rhs(u1)
            g2x, g2y = self._resistive(b1x, b1y)
            for q in range(6):
                self.A[q] = self.A[q] + f2[q] * self.c_1md
            self.A[4] = self.A[4] + g2x * self.c_1mg
            self.A[5] = self.A[5] + g2y * self.c_1mg

    def finalize(self):
        rx, ry = self._rate(self.x)
        b2x = self.A[4] + rx * self.c_g
        b2y = self.A[5] + ry * self.c_g
        g3x, g3y = self._resistive(b2x, b2y)
        self.S[4] = self.A[4] + g3x * self.c_g
        self.S[5] = self.A[5] + g3y * self.c_g
        self.S[0] = np.where(self.A[0] < RHO_FLOOR, RHO_FLOOR, self.A[0])
        for q in (1, 2, 3):
            self.S[q] = self.A[q].copy()

    # -- conjugate gradient on the interior corners (wait=False keeps the sums for sums())
    def sums(self, n):
        out, self._sums = self._sums, None
        assert out is not None and len(out) == n
        return out

    def _ret(self, vals, wait):
        if wait:
            return vals
        self._sums = vals
        return None

    def cg_rhs(self, index, wait=True):
        bx, by = (self.T[4], self.T[5]) if index == 0 else (self.A[4], self.A[5])
        I = self.I
        idx, idy = 1.0 / self.dx, 1.0 / self.dy
        b = self.eta * ((by - np.roll(by, 1, axis=1)) * idx - (bx - np.roll(bx, 1, axis=0)) * idy)
        self.r[I] = b[I]
        self.zv[I] = self.invdiag * b[I]
        self.p[I] = self.zv[I]
        self.x[I] = 0.0
        return self._ret([float(np.sum(b[I] * b[I])), float(np.sum(b[I] * self.zv[I]))], wait)

    def cg_matvec(self, wait=True):
        I, p = self.I, self.p
        q = (-self.cy) * np.roll(p, 1, axis=0) + (-self.cx) * np.roll(p, 1, axis=1) + self.diag * p + \
            (-self.cx) * np.roll(p, -1, axis=1) + (-self.cy) * np.roll(p, -1, axis=0)
        self.q[I] = q[I]
        return self._ret([float(np.sum(p[I] * q[I]))], wait)

    def cg_update(self, alpha, wait=True):
        I = self.I
        self.x[I] = self.x[I] + alpha * self.p[I]
        self.r[I] = self.r[I] - alpha * self.q[I]
        self.zv[I] = self.invdiag * self.r[I]
        return self._ret([float(np.sum(self.r[I] * self.r[I])), float(np.sum(self.r[I] * self.zv[I]))], wait)

    def cg_direction(self, beta):
        I = self.I
        self.p[I] = self.zv[I] + beta * self.p[I]

    def cg_zero_solution(self):
        self.x[self.I] = 0.0

    # -- the same phases with the decisions in a control block (slot: this subdomain's 4 sums,
    # ctl: the control block; both numpy arrays of a host decision group)
    def cg_rhs_dev(self, index, slot):
        slot[:2] = self.cg_rhs(index)

    def cg_matvec_dev(self, ctl, slot):
        if ctl[0] != 0.0:
            slot[0] = self.cg_matvec()[0]

    def cg_update_dev(self, ctl, slot):
        if ctl[0] != 0.0:
            slot[:2] = self.cg_update(float(ctl[6]))

    def cg_direction_dev(self, ctl):
        if ctl[0] != 0.0:
            self.cg_direction(float(ctl[7]))

    def cg_finish_dev(self, ctl):
        if ctl[1] == 2.0:  # non-finite
            self.cg_zero_solution()
