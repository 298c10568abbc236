"""torch.autograd binding of the adjoint C ABI (mhd_adj_*): a differentiable fixed-dt IMEX trajectory.

``trajectory(u0, eta, adj)`` maps an initial state u0 (a (6, ny, nx) float64 CUDA tensor in the
order rho, mx, my, E, bxf, byf) and the resistivity eta (a 0-dim float64 tensor) to the state after
``adj.nsteps`` steps of size ``adj.dt``; its backward runs the hand-written adjoint kernels (with
checkpointed recomputation) and returns dL/du0 and dL/deta. Torch supplies device memory and the
autograd graph only: every step and every adjoint step runs in libmhd_b200.so.

``state_from_potential`` builds u0 from a corner vector potential Az with torch operations
(benchmarks.hpp:58-62: face B = curl Az, E from the cell-averaged face B), so that gradients reach
Az through autograd.
"""
from __future__ import annotations

import torch

from .capi import Adjoint

GAMMA = 5.0 / 3.0


def _after_current_stream(adj: Adjoint, device: torch.device) -> None:
    """Order the library's stream after the work torch has queued on its current stream (that
    produced the inputs): an event, not a device-wide synchronisation. The library's calls return
    only when their own stream is done, so torch's later work needs no further ordering."""
    ev = torch.cuda.Event()
    ev.record(torch.cuda.current_stream(device))
    torch.cuda.ExternalStream(adj.stream, device=device).wait_event(ev)


def _ptrs(t: torch.Tensor):
    if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or t.dim() != 3 or t.shape[0] != 6:
        raise ValueError("states must be contiguous float64 CUDA tensors of shape (6, ny, nx)")
    return [t[k].data_ptr() for k in range(6)]


class _Trajectory(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0: torch.Tensor, eta: torch.Tensor, adj: Adjoint):
        u0c = u0.detach().contiguous()
        adj.set_eta(float(eta))
        uT = torch.empty_like(u0c)
        _after_current_stream(adj, u0c.device)  # the library runs on its own stream
        adj.forward(_ptrs(u0c), _ptrs(uT))
        adj._generation = getattr(adj, "_generation", 0) + 1
        ctx.adj = adj
        ctx.generation = adj._generation
        ctx.eta_shape = eta.shape
        return uT

    @staticmethod
    def backward(ctx, grad_uT: torch.Tensor):
        adj = ctx.adj
        if adj._generation != ctx.generation:
            raise RuntimeError("the Adjoint object ran another forward pass since this one; "
                               "use one Adjoint per trajectory in flight")
        g = grad_uT.detach().contiguous()
        gu0 = torch.empty_like(g)
        _after_current_stream(adj, g.device)
        geta = adj.backward(_ptrs(g), _ptrs(gu0))
        return gu0, torch.tensor(geta, dtype=torch.float64, device=g.device).reshape(ctx.eta_shape), None


def trajectory(u0: torch.Tensor, eta: torch.Tensor, adj: Adjoint) -> torch.Tensor:
    """State after adj.nsteps fixed-dt IMEX steps from u0 with resistivity eta (differentiable in
    both)."""
    return _Trajectory.apply(u0, eta, adj)


def _at(f, di, dj):
    return torch.roll(f, shifts=(-dj, -di), dims=(-2, -1))


def state_from_potential(az: torch.Tensor, rho: torch.Tensor, vx: torch.Tensor, vy: torch.Tensor,
                         p: torch.Tensor, dx: float, dy: float) -> torch.Tensor:
    """Conserved state (6, ny, nx) from the corner potential az (ny, nx; az[j, i] at the
    bottom-left corner of cell (i, j), periodic) and cell-centred rho, v, p:
    bxf = (Az(i, j+1) - Az(i, j))/dy, byf = -(Az(i+1, j) - Az(i, j))/dx (benchmarks.hpp:58-59),
    E = p/(gamma-1) + rho|v|^2/2 + |B_c|^2/2 with B_c the face averages (benchmarks.hpp:61-62)."""
    bx = (_at(az, 0, 1) - az) / dy
    by = -(_at(az, 1, 0) - az) / dx
    bxc = 0.5 * (bx + _at(bx, 1, 0))
    byc = 0.5 * (by + _at(by, 0, 1))
    E = p / (GAMMA - 1.0) + 0.5 * rho * (vx * vx + vy * vy) + 0.5 * (bxc * bxc + byc * byc)
    return torch.stack([rho, rho * vx, rho * vy, E, bx, by])
