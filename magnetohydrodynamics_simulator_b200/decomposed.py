"""Domain decomposition of one periodic grid into P x Q subdomains (the mhd_sub_* C ABI).

The reference grows one Grid on one thread (src/integrator_main.cpp:29-30); past one GPU's memory
the grid is split. Each subdomain is an ``mhd_subdomain`` on some GPU: its interior plus a ring of
``HALO`` cells. This module is the driver around them: the partition, the ring exchanges between
kernels, and the global reductions of the implicit solve and the CFL step.

* ``Partition``: subdomain sizes and offsets (the remainder of nx / P and ny / Q goes to the first
  columns / rows of subdomains) and the periodic neighbours; subdomain index = q * P + p.
* Transports move the rings and add the partial sums:
  - ``LocalTransport``: every subdomain in this process (one GPU, or a CPU stand-in in the tests):
    strips go from one subdomain's buffer into its neighbour's ring directly;
  - ``DistTransport``: one subdomain per rank of a ``torch.distributed`` process group (NCCL for
    GPU buffers, gloo for CPU ones): a ring exchange is two shifts per axis (each rank sends one
    strip and receives one), and partial sums are all-gathered and added in rank order, so every
    rank takes the same decisions.
* ``DecomposedRun``: one ARS(2,2,2) step over the subdomains (solvers.hpp:491-613): the explicit
  kernels on the extended planes, ring exchanges between them, and the implicit solves as a
  conjugate gradient with Eigen's rules (x0 = 0, Jacobi scaling, stop when
  |r|^2 < max(tol^2 |b|^2, DBL_MIN), at most 2 n products) whose dot products are sums of the
  subdomains' partials in a fixed order. dt is the CFL step of diagnostics.hpp:82-84 from the
  largest interior signal speed of all subdomains.

A subdomain object needs: set_state, get_state, pack(set, side, width) -> buffer,
unpack(set, side, width, buffer), synchronize, cfl_speed, set_step, stage(1|2), finalize,
cg_rhs, cg_matvec, cg_update (each with wait=False: enqueue only, sums(n) returns the sums),
cg_direction, cg_zero_solution, divb_sums; and, where its work runs on a stream, record_event /
wait_event, with which LocalTransport orders the subdomains' streams without host waits.
``GpuSubdomain`` is the one over the C ABI.

The solve's decisions can stay on the device (``device_decisions``): the subdomains' phases
(cg_rhs_dev, cg_matvec_dev, cg_update_dev, cg_direction_dev, cg_finish_dev) write their sums into
a group's slots and read alpha and beta from its control block (``DeviceCgGroup``, mhd_subcg_* of
the C ABI; ``HostCgGroup`` applies the same rules to host arrays for CPU stand-ins), and the host
polls the control block one product behind instead of waiting for every phase's sums. The results
are bit-identical to the host decisions.
"""
from __future__ import annotations

import ctypes
import math
from typing import List, Sequence

import numpy as np

from .capi import MHDError, Params, _check, load_library

HALO = 4
WEST, EAST, SOUTH, NORTH = 0, 1, 2, 3
OPPOSITE = {WEST: EAST, EAST: WEST, SOUTH: NORTH, NORTH: SOUTH}
SET_STATE, SET_PREDICTOR, SET_ACCUMULATOR_B, SET_SOLUTION, SET_DIRECTION = 0, 1, 2, 3, 4
SET_CG_EVEN, SET_CG_ODD = 5, 6  # the single-sweep solve's r_k and p_{k-1}
DBL_MIN = 2.2250738585072014e-308
EPS = 2.220446049250313e-16
ARS_G = (2.0 - math.sqrt(2.0)) / 2.0  # solvers.hpp:41
# control block of the device-resident decisions (MHD_SUBCG_* of include/mhd_b200.h)
SUBCG_CTL = 16
CG_ACTIVE, CG_STATUS, CG_PRODUCTS, CG_ALPHA, CG_BETA = 0, 1, 2, 6, 7
CG_DT, CG_CFL_NONFINITE = 14, 15
CG_OK, CG_NOT_CONVERGED, CG_NONFINITE = 0, 1, 2


class Partition:
    """P x Q blocks of an nx x ny periodic grid."""

    def __init__(self, nx: int, ny: int, P: int, Q: int):
        if P < 1 or Q < 1 or nx // P < HALO or ny // Q < HALO:
            raise ValueError(f"every subdomain needs at least {HALO} x {HALO} cells")
        self.nx, self.ny, self.P, self.Q = nx, ny, P, Q

        def split(n, k):
            sizes = [n // k + (1 if i < n % k else 0) for i in range(k)]
            offs = [sum(sizes[:i]) for i in range(k)]
            return sizes, offs

        self.xs, self.x0 = split(nx, P)
        self.ys, self.y0 = split(ny, Q)

    @property
    def count(self) -> int:
        return self.P * self.Q

    def coords(self, idx: int):
        return idx % self.P, idx // self.P

    def shape(self, idx: int):
        p, q = self.coords(idx)
        return self.xs[p], self.ys[q]  # (nx, ny) of the interior

    def window(self, idx: int):
        """(row slice, column slice) of the subdomain's interior in the global arrays."""
        p, q = self.coords(idx)
        return slice(self.y0[q], self.y0[q] + self.ys[q]), slice(self.x0[p], self.x0[p] + self.xs[p])

    def neighbour(self, idx: int, side: int) -> int:
        p, q = self.coords(idx)
        if side == WEST:
            p = (p - 1) % self.P
        elif side == EAST:
            p = (p + 1) % self.P
        elif side == SOUTH:
            q = (q - 1) % self.Q
        else:
            q = (q + 1) % self.Q
        return q * self.P + p


class GpuSubdomain:
    """One subdomain on the current CUDA device (mhd_sub_* of the C ABI)."""

    def __init__(self, nx: int, ny: int, dx: float, dy: float, eta: float, *, ct_mode: int = 0,
                 stream: int | None = None):
        import torch

        self.torch = torch
        self.lib = _bind(load_library())
        self.nx, self.ny = int(nx), int(ny)
        p = Params()
        _check(self.lib.mhd_default_params(ctypes.byref(p), nx, ny, dx, dy, eta), "mhd_default_params")
        p.ct_mode = ct_mode
        h = ctypes.c_void_p()
        _check(self.lib.mhd_sub_create(ctypes.byref(p), ctypes.c_void_p(stream) if stream else None,
                                       ctypes.byref(h)), "mhd_sub_create")
        self.h = h
        self._bufs = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_sub_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return self.lib.mhd_sub_stream(self.h) or 0

    def set_state(self, fields: Sequence[np.ndarray]):
        fs = [np.ascontiguousarray(f, dtype=np.float64) for f in fields]
        arr = (ctypes.c_void_p * 6)(*[f.ctypes.data for f in fs])
        _check(self.lib.mhd_sub_set_state(self.h, arr), "mhd_sub_set_state")

    def get_state(self):
        out = [np.empty((self.ny, self.nx)) for _ in range(6)]
        arr = (ctypes.c_void_p * 6)(*[f.ctypes.data for f in out])
        _check(self.lib.mhd_sub_get_state(self.h, arr), "mhd_sub_get_state")
        return out

    def _buffer(self, key, n):
        b = self._bufs.get(key)
        if b is None or b.numel() != n:
            b = self.torch.empty(n, dtype=self.torch.float64, device="cuda")
            self._bufs[key] = b
        return b

    def pack(self, set_: int, side: int, width: int):
        n = self.lib.mhd_sub_strip_doubles(self.h, set_, side, width)
        buf = self._buffer((set_, side, width), n)
        _check(self.lib.mhd_sub_pack(self.h, set_, side, width, ctypes.c_void_p(buf.data_ptr())), "mhd_sub_pack")
        return buf

    def recv_buffer(self, set_: int, side: int, width: int):
        n = self.lib.mhd_sub_strip_doubles(self.h, set_, side, width)
        return self._buffer(("recv", set_, side, width), n)

    def unpack(self, set_: int, side: int, width: int, buf):
        _check(self.lib.mhd_sub_unpack(self.h, set_, side, width, ctypes.c_void_p(buf.data_ptr())),
               "mhd_sub_unpack")

    def synchronize(self):
        _check(self.lib.mhd_sub_synchronize(self.h), "mhd_sub_synchronize")

    # stream ordering between subdomains (rings move without host waits)
    def record_event(self):
        ev = self.torch.cuda.Event()
        ev.record(self.torch.cuda.ExternalStream(self.stream))
        return ev

    def wait_event(self, ev):
        if ev is not None:
            self.torch.cuda.ExternalStream(self.stream).wait_event(ev)

    def cfl_speed(self):
        v, bad = ctypes.c_double(), ctypes.c_int()
        _check(self.lib.mhd_sub_cfl_speed(self.h, ctypes.byref(v), ctypes.byref(bad)), "mhd_sub_cfl_speed")
        return v.value, bool(bad.value)

    def set_step(self, dt: float, alpha: float):
        _check(self.lib.mhd_sub_set_step(self.h, dt, alpha), "mhd_sub_set_step")

    def stage(self, k: int):
        _check(self.lib.mhd_sub_stage(self.h, k), "mhd_sub_stage")

    def finalize(self):
        _check(self.lib.mhd_sub_finalize(self.h), "mhd_sub_finalize")

    # CG phases: wait=True returns the phase's sums; wait=False only enqueues (sums() reads them)
    def cg_rhs(self, solve_index: int, wait: bool = True):
        out = (ctypes.c_double * 2)() if wait else None
        _check(self.lib.mhd_sub_cg_rhs(self.h, solve_index, out), "mhd_sub_cg_rhs")
        return [out[0], out[1]] if wait else None

    def cg_matvec(self, wait: bool = True):
        v = ctypes.c_double() if wait else None
        _check(self.lib.mhd_sub_cg_matvec(self.h, ctypes.byref(v) if wait else None), "mhd_sub_cg_matvec")
        return [v.value] if wait else None

    def cg_update(self, alpha: float, wait: bool = True):
        out = (ctypes.c_double * 2)() if wait else None
        _check(self.lib.mhd_sub_cg_update(self.h, alpha, out), "mhd_sub_cg_update")
        return [out[0], out[1]] if wait else None

    def sums(self, n: int):
        out = (ctypes.c_double * n)()
        _check(self.lib.mhd_sub_sums(self.h, out, n), "mhd_sub_sums")
        return list(out)

    def cg_direction(self, beta: float):
        _check(self.lib.mhd_sub_cg_direction(self.h, beta), "mhd_sub_cg_direction")

    def cg_zero_solution(self):
        _check(self.lib.mhd_sub_cg_zero_solution(self.h), "mhd_sub_cg_zero_solution")

    def divb_sums(self):
        out = (ctypes.c_double * 2)()
        _check(self.lib.mhd_sub_divb_sums(self.h, out), "mhd_sub_divb_sums")
        return [out[0], out[1]]

    # CG phases with the decisions on the device: slot and ctl are device addresses (ints)
    def cg_rhs_dev(self, solve_index: int, slot: int):
        _check(self.lib.mhd_sub_cg_rhs_dev(self.h, solve_index, slot), "mhd_sub_cg_rhs_dev")

    def cg_matvec_dev(self, ctl: int, slot: int):
        _check(self.lib.mhd_sub_cg_matvec_dev(self.h, ctl, slot), "mhd_sub_cg_matvec_dev")

    def cg_update_dev(self, ctl: int, slot: int):
        _check(self.lib.mhd_sub_cg_update_dev(self.h, ctl, slot), "mhd_sub_cg_update_dev")

    def cg_direction_dev(self, ctl: int):
        _check(self.lib.mhd_sub_cg_direction_dev(self.h, ctl), "mhd_sub_cg_direction_dev")

    def cg_finish_dev(self, ctl: int):
        _check(self.lib.mhd_sub_cg_finish_dev(self.h, ctl), "mhd_sub_cg_finish_dev")

    # the single-sweep form of the solve (the single context's sweeps on the interior)
    def cg_sweep_rhs_dev(self, solve_index: int, slot: int):
        _check(self.lib.mhd_sub_cg_sweep_rhs_dev(self.h, solve_index, slot), "mhd_sub_cg_sweep_rhs_dev")

    def cg_sweep_iter_dev(self, ctl: int, slot: int):
        _check(self.lib.mhd_sub_cg_sweep_iter_dev(self.h, ctl, slot), "mhd_sub_cg_sweep_iter_dev")

    def cg_sweep_finish_dev(self, ctl: int):
        _check(self.lib.mhd_sub_cg_sweep_finish_dev(self.h, ctl), "mhd_sub_cg_sweep_finish_dev")


class DeviceCgGroup:
    """The decisions of one decomposed solve on the device (mhd_subcg of the C ABI): a control
    block and `count` sum slots. `slots`: a CUDA tensor of count * 4 doubles to use as the slots
    (across ranks, where they are all-gathered), else the group allocates them."""

    def __init__(self, lib, count: int, stream: int, slots=None):
        self.lib = lib
        self.count = count
        self._slots_tensor = slots
        h = ctypes.c_void_p()
        _check(lib.mhd_subcg_create(count, ctypes.c_void_p(stream) if stream else None,
                                    ctypes.c_void_p(slots.data_ptr()) if slots is not None else None,
                                    ctypes.byref(h)), "mhd_subcg_create")
        self.h = h
        self.slots = lib.mhd_subcg_slots(h)
        self.ctl = lib.mhd_subcg_control(h)

    def slot(self, i: int) -> int:
        return self.slots + 32 * i

    def decide(self, phase: int, tol: float, max_products: int):
        """On the group's stream (the subdomain shares it, or the caller orders them)."""
        _check(self.lib.mhd_subcg_decide(self.h, phase, tol, max_products), "mhd_subcg_decide")

    def decide_on(self, handles, phase: int, tol: float, max_products: int):
        """Ordered by events after the subdomains' work so far, and their later work after it."""
        _check(self.lib.mhd_subcg_decide_on(self.h, handles, phase, tol, max_products), "mhd_subcg_decide_on")

    def product(self, handles, P: int, Q: int, tol: float, max_products: int, tag: int):
        """One product of the solve on the P x Q subdomains as a replayed CUDA graph; posts `tag`."""
        _check(self.lib.mhd_subcg_product(self.h, handles, P, Q, tol, max_products, tag), "mhd_subcg_product")

    def sweep_product(self, handles, P: int, Q: int, tol: float, max_products: int, k: int, tag: int):
        """Iteration k of the single-sweep solve as a replayed CUDA graph; posts `tag`."""
        _check(self.lib.mhd_subcg_sweep_product(self.h, handles, P, Q, tol, max_products, k, tag),
               "mhd_subcg_sweep_product")

    def cfl_step(self, handles, courant: float, safety: float):
        """The CFL step of all subdomains and their step coefficients, on the device."""
        _check(self.lib.mhd_subcg_cfl_step(self.h, handles, courant, safety), "mhd_subcg_cfl_step")

    def post(self, tag: int):
        _check(self.lib.mhd_subcg_post(self.h, tag), "mhd_subcg_post")

    def read(self, tag: int):
        out = (ctypes.c_double * SUBCG_CTL)()
        _check(self.lib.mhd_subcg_read(self.h, tag, out), "mhd_subcg_read")
        return list(out)

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_subcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostCgGroup:
    """The same control block and slots in host memory, for CPU stand-in subdomains; the rules are
    the library's (mhd_subcg_decide_host)."""

    def __init__(self, lib, count: int):
        self.lib = lib
        self.count = count
        self.ctl = np.zeros(SUBCG_CTL)
        self.slots = np.zeros(4 * count)
        self._posted = [None] * 4

    def slot(self, i: int):
        return self.slots[4 * i:4 * i + 4]

    def decide(self, phase: int, tol: float, max_products: int):
        dp = ctypes.POINTER(ctypes.c_double)
        _check(self.lib.mhd_subcg_decide_host(self.ctl.ctypes.data_as(dp), self.slots.ctypes.data_as(dp),
                                              self.count, phase, tol, max_products), "mhd_subcg_decide_host")

    def post(self, tag: int):
        self._posted[tag % 4] = self.ctl.copy()

    def read(self, tag: int):
        return [float(v) for v in self._posted[tag % 4]]

    def close(self):
        pass


_bound = set()


def _bind(lib):
    if id(lib) in _bound:
        return lib
    vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    ip = ctypes.c_int
    lib.mhd_sub_halo.restype = ip
    lib.mhd_sub_create.argtypes = [ctypes.POINTER(Params), vp, ctypes.POINTER(vp)]
    lib.mhd_sub_destroy.argtypes = [vp]
    lib.mhd_sub_stream.argtypes = [vp]
    lib.mhd_sub_stream.restype = vp
    lib.mhd_sub_set_state.argtypes = [vp, ctypes.POINTER(vp)]
    lib.mhd_sub_get_state.argtypes = [vp, ctypes.POINTER(vp)]
    lib.mhd_sub_strip_doubles.argtypes = [vp, ip, ip, ip]
    lib.mhd_sub_strip_doubles.restype = ctypes.c_size_t
    lib.mhd_sub_pack.argtypes = [vp, ip, ip, ip, vp]
    lib.mhd_sub_unpack.argtypes = [vp, ip, ip, ip, vp]
    lib.mhd_sub_cfl_speed.argtypes = [vp, dp, ctypes.POINTER(ip)]
    lib.mhd_sub_set_step.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    lib.mhd_sub_stage.argtypes = [vp, ip]
    lib.mhd_sub_finalize.argtypes = [vp]
    lib.mhd_sub_cg_rhs.argtypes = [vp, ip, dp]
    lib.mhd_sub_cg_matvec.argtypes = [vp, dp]
    lib.mhd_sub_cg_update.argtypes = [vp, ctypes.c_double, dp]
    lib.mhd_sub_cg_direction.argtypes = [vp, ctypes.c_double]
    lib.mhd_sub_cg_zero_solution.argtypes = [vp]
    lib.mhd_sub_divb_sums.argtypes = [vp, dp]
    lib.mhd_sub_synchronize.argtypes = [vp]
    lib.mhd_sub_sums.argtypes = [vp, dp, ip]
    lib.mhd_sub_exchange_local.argtypes = [ctypes.POINTER(vp), ip, ip, ip, ip]
    lib.mhd_sub_cg_rhs_dev.argtypes = [vp, ip, vp]
    lib.mhd_sub_cg_matvec_dev.argtypes = [vp, vp, vp]
    lib.mhd_sub_cg_update_dev.argtypes = [vp, vp, vp]
    lib.mhd_sub_cg_direction_dev.argtypes = [vp, vp]
    lib.mhd_sub_cg_finish_dev.argtypes = [vp, vp]
    lib.mhd_subcg_create.argtypes = [ip, vp, vp, ctypes.POINTER(vp)]
    lib.mhd_subcg_destroy.argtypes = [vp]
    lib.mhd_subcg_slots.argtypes = [vp]
    lib.mhd_subcg_slots.restype = ctypes.c_size_t
    lib.mhd_subcg_control.argtypes = [vp]
    lib.mhd_subcg_control.restype = ctypes.c_size_t
    lib.mhd_subcg_decide.argtypes = [vp, ip, ctypes.c_double, ctypes.c_longlong]
    lib.mhd_subcg_post.argtypes = [vp, ip]
    lib.mhd_subcg_read.argtypes = [vp, ip, dp]
    lib.mhd_subcg_decide_host.argtypes = [dp, dp, ip, ip, ctypes.c_double, ctypes.c_longlong]
    lib.mhd_subcg_decide_on.argtypes = [vp, ctypes.POINTER(vp), ip, ctypes.c_double, ctypes.c_longlong]
    lib.mhd_subcg_product.argtypes = [vp, ctypes.POINTER(vp), ip, ip, ctypes.c_double, ctypes.c_longlong, ip]
    lib.mhd_subcg_sweep_product.argtypes = [vp, ctypes.POINTER(vp), ip, ip, ctypes.c_double, ctypes.c_longlong,
                                            ip, ip]
    lib.mhd_subcg_cfl_step.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_double, ctypes.c_double]
    lib.mhd_sub_cg_sweep_rhs_dev.argtypes = [vp, ip, vp]
    lib.mhd_sub_cg_sweep_iter_dev.argtypes = [vp, vp, vp]
    lib.mhd_sub_cg_sweep_finish_dev.argtypes = [vp, vp]
    assert lib.mhd_sub_halo() == HALO
    _bound.add(id(lib))
    return lib


def _ordered_sum(rows) -> List[float]:
    """Add equal-length lists of partial sums in the given order (subdomain / rank order)."""
    out = [0.0] * len(rows[0])
    for r in rows:
        for k, v in enumerate(r):
            out[k] += float(v)
    return out


class LocalTransport:
    """Every subdomain in this process; `subs[i]` is subdomain i of the partition."""

    def __init__(self, part: Partition, subs: Sequence, native: bool = True):
        assert len(subs) == part.count
        self.part = part
        self.subs = list(subs)
        # GPU subdomains of one process exchange natively (device copies ordered by events);
        # native=False moves their strips through pack/unpack buffers, as across GPUs
        self._native = None
        self._handles = None
        if all(isinstance(s_, GpuSubdomain) for s_ in self.subs):
            self._handles = (ctypes.c_void_p * part.count)(*[s_.h for s_ in self.subs])
            if native:
                self._native = self._handles

    @property
    def own(self):
        return self.subs

    def exchange(self, set_: int, width: int):
        """Both axes, west/east then south/north. GPU subdomains use mhd_sub_exchange_local (direct
        device copies, ordered by events). Other subdomains with streams (record_event) pack and
        unpack through buffers ordered by events; the rest run in call order."""
        if self._native is not None:
            _check(self.subs[0].lib.mhd_sub_exchange_local(self._native, self.part.P, self.part.Q,
                                                           set_, width), "mhd_sub_exchange_local")
            return
        evented = hasattr(self.subs[0], "record_event")
        if not hasattr(self, "_consumed"):
            self._consumed = {}
        for axis in ((EAST, WEST), (NORTH, SOUTH)):
            bufs, packed = {}, {}
            for i, s in enumerate(self.subs):
                for side in axis:
                    if evented:
                        s.wait_event(self._consumed.get((i, set_, side, width)))
                    bufs[(i, side)] = s.pack(set_, side, width)
                    if evented:
                        packed[(i, side)] = s.record_event()
            for i, s in enumerate(self.subs):
                for side in axis:
                    nb = self.part.neighbour(i, side)
                    if evented:
                        s.wait_event(packed[(nb, OPPOSITE[side])])
                    s.unpack(set_, side, width, bufs[(nb, OPPOSITE[side])])
                    if evented:
                        self._consumed[(nb, set_, OPPOSITE[side], width)] = s.record_event()

    def sum(self, rows) -> List[float]:
        return _ordered_sum(rows)

    def max(self, values) -> float:
        return max(values)

    def any(self, flags) -> bool:
        return any(flags)

    # device-resident decisions: every subdomain writes its own slot of one group
    def cg_group(self):
        """A decision group for the subdomains, or None where the host must decide: GPU
        subdomains get a DeviceCgGroup on a stream of its own (ordered against theirs by events),
        CPU stand-ins a HostCgGroup."""
        gpu = [isinstance(s_, GpuSubdomain) for s_ in self.subs]
        if all(gpu):
            return DeviceCgGroup(self.subs[0].lib, self.part.count, 0)
        if not any(gpu):
            return HostCgGroup(_bind(load_library()), self.part.count)
        return None

    def own_slots(self, group):
        return [group.slot(i) for i in range(self.part.count)]

    def gather_slots(self, group):
        pass


class DistTransport:
    """One subdomain per rank of the default torch.distributed group (rank = subdomain index).
    GPU subdomains exchange CUDA tensors (NCCL); CPU stand-ins exchange CPU tensors (gloo)."""

    def __init__(self, part: Partition, sub, device=None):
        import torch
        import torch.distributed as dist

        self.torch, self.dist = torch, dist
        self.part = part
        self.rank = dist.get_rank()
        assert dist.get_world_size() == part.count
        self.sub = sub
        self.device = device if device is not None else torch.device("cpu")

    @property
    def own(self):
        return [self.sub]

    def _as_tensor(self, buf):
        if isinstance(buf, np.ndarray):
            return self.torch.from_numpy(np.ascontiguousarray(buf))
        return buf

    def exchange(self, set_: int, width: int):
        if isinstance(self.sub, GpuSubdomain):
            return self._exchange_stream_ordered(set_, width)
        for axis in ((EAST, WEST), (NORTH, SOUTH)):
            for side in axis:
                # shift toward `side`: send this side's strip to that neighbour, receive the strip
                # the opposite neighbour sent toward `side` into the opposite ring
                send = self.sub.pack(set_, side, width)
                self.sub.synchronize()
                dst = self.part.neighbour(self.rank, side)
                src = self.part.neighbour(self.rank, OPPOSITE[side])
                if dst == self.rank:
                    self.sub.unpack(set_, OPPOSITE[side], width, send)
                    continue
                st = self._as_tensor(send)
                rt = self.torch.empty_like(st)
                ops = [self.dist.P2POp(self.dist.isend, st, dst), self.dist.P2POp(self.dist.irecv, rt, src)]
                for req in self.dist.batch_isend_irecv(ops):
                    req.wait()
                if rt.is_cuda:
                    # wait() orders torch's current stream after the transfer; the unpack runs on
                    # the subdomain's own stream, so finish the transfer first
                    self.torch.cuda.current_stream().synchronize()
                self.sub.unpack(set_, OPPOSITE[side], width, rt.numpy() if isinstance(send, np.ndarray) else rt)
            self.sub.synchronize()

    def _exchange_stream_ordered(self, set_: int, width: int):
        """The same shifts for a GPU subdomain with every step on its stream: pack, the NCCL
        transfer (issued with the subdomain's stream as torch's current stream, which then waits
        for it) and unpack follow one another on the device without a host wait. The strips travel
        in the subdomain's persistent pack and receive buffers."""
        torch = self.torch
        with torch.cuda.stream(torch.cuda.ExternalStream(self.sub.stream)):
            for axis in ((EAST, WEST), (NORTH, SOUTH)):
                for side in axis:
                    send = self.sub.pack(set_, side, width)
                    dst = self.part.neighbour(self.rank, side)
                    src = self.part.neighbour(self.rank, OPPOSITE[side])
                    if dst == self.rank:
                        self.sub.unpack(set_, OPPOSITE[side], width, send)
                        continue
                    recv = self.sub.recv_buffer(set_, OPPOSITE[side], width)
                    ops = [self.dist.P2POp(self.dist.isend, send, dst), self.dist.P2POp(self.dist.irecv, recv, src)]
                    for req in self.dist.batch_isend_irecv(ops):
                        req.wait()
                    self.sub.unpack(set_, OPPOSITE[side], width, recv)

    def _gather(self, values) -> np.ndarray:
        t = self.torch.tensor(values, dtype=self.torch.float64, device=self.device)
        out = self.torch.empty(self.part.count * t.numel(), dtype=self.torch.float64, device=self.device)
        self.dist.all_gather_into_tensor(out, t)
        return out.cpu().numpy().reshape(self.part.count, -1)

    def sum(self, rows) -> List[float]:
        (mine,) = rows
        return _ordered_sum(list(self._gather(list(mine))))

    def max(self, values) -> float:
        (mine,) = values
        return float(np.max(self._gather([mine])))

    def any(self, flags) -> bool:
        (mine,) = flags
        return bool(np.any(self._gather([1.0 if mine else 0.0])))

    # device-resident decisions: this rank's sums go into a local slot, all-gathered into the
    # group's slots in rank order before every decision
    def cg_group(self):
        torch = self.torch
        if isinstance(self.sub, GpuSubdomain):
            self._slots = torch.zeros(4 * self.part.count, dtype=torch.float64, device="cuda")
            self._local = torch.zeros(4, dtype=torch.float64, device="cuda")
            return DeviceCgGroup(self.sub.lib, self.part.count, self.sub.stream, slots=self._slots)
        self._local = np.zeros(4)
        return HostCgGroup(_bind(load_library()), self.part.count)

    def own_slots(self, group):
        return [self._local.data_ptr() if isinstance(group, DeviceCgGroup) else self._local]

    def gather_slots(self, group):
        torch = self.torch
        if isinstance(group, DeviceCgGroup):
            # on the subdomain's stream: the collective follows its phase and precedes the decision
            with torch.cuda.stream(torch.cuda.ExternalStream(self.sub.stream)):
                self.dist.all_gather_into_tensor(self._slots, self._local)
            return
        out = torch.empty(4 * self.part.count, dtype=torch.float64)
        self.dist.all_gather_into_tensor(out, torch.from_numpy(self._local))
        group.slots[:] = out.numpy()


class DecomposedRun:
    """ARS(2,2,2) steps of one nx x ny periodic grid split over the transport's subdomains."""

    def __init__(self, part: Partition, transport, dx: float, dy: float, eta: float, *,
                 courant: float = 0.5, safety: float = 0.9, cg_tol: float = 0.0, cg_max_iters: int = 0,
                 device_decisions: bool = True, cg_form: str | None = None, poll_lag: int = 1):
        """device_decisions: take the solve's decisions on the device (DeviceCgGroup) where the
        transport allows it; False keeps them on the host (both give bit-identical results).
        cg_form: "sweep", the single context's single-sweep solver on every subdomain (GPU
        subdomains with device decisions; the default there), or "two_sweep" (a matrix product
        and an update per product; every other case). poll_lag (1-3): with device decisions the
        host reads the control block posted poll_lag iterations back, so that many iterations
        stay queued (each solve then runs poll_lag no-op iterations after its end)."""
        if not 1 <= poll_lag <= 3:
            raise ValueError("poll_lag must be 1, 2 or 3")
        self.poll_lag = poll_lag
        self.part, self.tr = part, transport
        self._group = transport.cg_group() if device_decisions else None
        self._slots = transport.own_slots(self._group) if self._group is not None else None
        sweep_ok = isinstance(self._group, DeviceCgGroup)
        if cg_form is None:
            cg_form = "sweep" if sweep_ok else "two_sweep"
        if cg_form not in ("sweep", "two_sweep") or (cg_form == "sweep" and not sweep_ok):
            raise ValueError(f"cg_form {cg_form!r} needs GPU subdomains with device decisions")
        self.cg_form = cg_form
        self.dx, self.dy, self.eta = dx, dy, eta
        self.courant, self.safety = courant, safety
        self.tol = cg_tol if cg_tol > 0 else EPS
        self.max_iters = cg_max_iters if cg_max_iters > 0 else 2 * part.nx * part.ny
        self.status = "ok"
        self.last_products = (0, 0)
        self._last_ctl = None

    def _own_indices(self):
        if isinstance(self.tr, LocalTransport):
            return list(range(self.part.count))
        return [self.tr.rank]

    def set_state(self, fields: Sequence[np.ndarray]):
        """Global dense (ny, nx) planes; each subdomain takes its window, then the rings fill."""
        for i, s in zip(self._own_indices(), self.tr.own):
            rs, cs = self.part.window(i)
            s.set_state([np.ascontiguousarray(f[rs, cs]) for f in fields])
        self.tr.exchange(SET_STATE, HALO)

    def get_state(self):
        """Global dense planes (every rank's interiors; with DistTransport gathered to all)."""
        out = [np.zeros((self.part.ny, self.part.nx)) for _ in range(6)]
        if isinstance(self.tr, LocalTransport):
            for i, s in enumerate(self.tr.subs):
                rs, cs = self.part.window(i)
                for k, f in enumerate(s.get_state()):
                    out[k][rs, cs] = f
            return out
        mine = np.stack(self.tr.sub.get_state())
        pieces = [None] * self.part.count
        self.tr.dist.all_gather_object(pieces, mine)
        for i, st in enumerate(pieces):
            rs, cs = self.part.window(i)
            for k in range(6):
                out[k][rs, cs] = st[k]
        return out

    def cfl_dt(self) -> float:
        """diagnostics.hpp:82-84 from the largest interior signal speed (the device formula)."""
        speeds, bad = zip(*[s.cfl_speed() for s in self.tr.own])
        if self.tr.any(list(bad)):
            self.status = "nonfinite"
        smaxv = max(self.tr.max(list(speeds)), 1e-8)
        hmin = min(self.dx, self.dy)
        dt_res = math.inf if self.eta == 0.0 else hmin * hmin / (4.0 * self.eta)
        dt_hyp = self.courant * hmin / smaxv
        return (dt_res if dt_res < dt_hyp else dt_hyp) * self.safety

    @staticmethod
    def _phase(own, launch, n):
        """Enqueue a CG phase on every subdomain first, then read their sums (in order)."""
        for s in own:
            launch(s)
        return [s.sums(n) for s in own]

    def _solve(self, index: int) -> int:
        if self._group is not None:
            return self._solve_device(index, self.cg_form == "sweep")
        own = self.tr.own
        bb, abs_new = self.tr.sum(self._phase(own, lambda s: s.cg_rhs(index, wait=False), 2))
        threshold = max(self.tol * self.tol * bb, DBL_MIN)
        if not math.isfinite(bb):
            self.status = "nonfinite"
            return 0
        if bb == 0.0 or bb < threshold:
            return 0  # x = 0 (cg_rhs zeroed it)
        products = 0
        converged = False
        for _ in range(self.max_iters):
            self.tr.exchange(SET_DIRECTION, 1)
            (pq,) = self.tr.sum(self._phase(own, lambda s: s.cg_matvec(wait=False), 1))
            alpha = abs_new / pq
            rr, rz = self.tr.sum(self._phase(own, lambda s: s.cg_update(alpha, wait=False), 2))
            products += 1
            if not (math.isfinite(rr) and math.isfinite(alpha)):
                self.status = "nonfinite"
                for s in own:
                    s.cg_zero_solution()
                return products
            if rr < threshold:
                converged = True
                break
            beta = rz / abs_new
            abs_new = rz
            for s in own:
                s.cg_direction(beta)
        if not converged:
            self.status = "cg_not_converged"
        return products

    def _solve_device(self, index: int, sweep: bool = False) -> int:
        """The solve with the decisions in the group's control block: each product is enqueued
        before the previous one's state is read back, so the host waits only for work that is
        already behind the device's queue; a product enqueued after the solve ended does nothing
        but its ring exchange. GPU subdomains of one process run each product as one replayed
        CUDA graph (mhd_subcg_product, mhd_subcg_sweep_product). sweep: the single-sweep form."""
        g, own, slots, tr = self._group, self.tr.own, self._slots, self.tr
        ctl = g.ctl
        maxp, tol = self.max_iters, self.tol
        handles = getattr(tr, "_handles", None) if isinstance(g, DeviceCgGroup) else None
        if handles is not None:
            def decide(phase):
                g.decide_on(handles, phase, tol, maxp)
        else:
            def decide(phase):
                tr.gather_slots(g)
                g.decide(phase, tol, maxp)
        graph = handles is not None and getattr(tr, "_native", None) is not None
        if sweep:
            return self._sweep_solve(index, g, own, slots, decide, graph, handles)
        for s, sl in zip(own, slots):
            s.cg_rhs_dev(index, sl)
        decide(0)
        tag = 0
        g.post(tag)
        for _ in range(maxp):
            tag += 1
            if graph:
                g.product(handles, self.part.P, self.part.Q, tol, maxp, tag)
            else:
                tr.exchange(SET_DIRECTION, 1)
                for s, sl in zip(own, slots):
                    s.cg_matvec_dev(ctl, sl)
                decide(1)
                for s, sl in zip(own, slots):
                    s.cg_update_dev(ctl, sl)
                decide(2)
                for s in own:
                    s.cg_direction_dev(ctl)
                g.post(tag)
            if tag < self.poll_lag:
                continue
            c = g.read(tag - self.poll_lag)
            if c[CG_ACTIVE] == 0.0:
                break  # the solve ended: later iterations change nothing in the control block
        else:
            c = g.read(tag)
        self._last_ctl = c
        for s in own:
            s.cg_finish_dev(ctl)
        st = int(c[CG_STATUS])
        if st == CG_NONFINITE:
            self.status = "nonfinite"
        elif st == CG_NOT_CONVERGED:
            self.status = "cg_not_converged"
        return int(c[CG_PRODUCTS])

    def _sweep_solve(self, index, g, own, slots, decide, graph, handles) -> int:
        """The single-sweep form of _solve_device: the right-hand side sweep and decision 3,
        then per iteration the sweep (reading the cells around each interior from the
        neighbours in the graphs, from the exchanged rings otherwise) and decision 4."""
        ctl, maxp, tol = g.ctl, self.max_iters, self.tol
        for s, sl in zip(own, slots):
            s.cg_sweep_rhs_dev(index, sl)
        decide(3)
        tag = 0
        g.post(tag)
        for k in range(maxp):
            tag += 1
            if graph:
                g.sweep_product(handles, self.part.P, self.part.Q, tol, maxp, k, tag)
            else:
                self.tr.exchange(SET_CG_ODD if k & 1 else SET_CG_EVEN, 2)
                for s, sl in zip(own, slots):
                    s.cg_sweep_iter_dev(ctl, sl)
                decide(4)
                g.post(tag)
            if tag < self.poll_lag:
                continue
            c = g.read(tag - self.poll_lag)
            if c[CG_ACTIVE] == 0.0:
                break  # the solve ended: later iterations change nothing in the control block
        else:
            c = g.read(tag)
        self._last_ctl = c
        for s in own:
            s.cg_sweep_finish_dev(ctl)
        st = int(c[CG_STATUS])
        if st == CG_NONFINITE:
            self.status = "nonfinite"
        elif st == CG_NOT_CONVERGED:
            self.status = "cg_not_converged"
        return int(c[CG_PRODUCTS])

    def close(self):
        """Release the decision group (the subdomains belong to the caller)."""
        if self._group is not None:
            self._group.close()
            self._group = None

    def step(self, dt: float = 0.0, alpha: float | None = None):
        """One IMEX step; dt <= 0 takes the CFL step. alpha defaults to (dt * eta) * g (the matrix
        the reference driver builds for this dt). Returns (dt, (products of the two solves))."""
        own = self.tr.own
        handles = getattr(self.tr, "_handles", None)
        device_cfl = (dt <= 0.0 and alpha is None and isinstance(self._group, DeviceCgGroup)
                      and handles is not None)
        if device_cfl:
            # dt and the step's coefficients on the device; dt comes back with the solve's polls
            self._group.cfl_step(handles, self.courant, self.safety)
        else:
            if dt <= 0.0:
                dt = self.cfl_dt()
            if alpha is None:
                alpha = (dt * self.eta) * ARS_G
            for s in own:
                s.set_step(dt, alpha)
        for s in own:
            s.stage(1)
        self.tr.exchange(SET_PREDICTOR, HALO)
        k1 = self._solve(0)
        self.tr.exchange(SET_SOLUTION, HALO)
        for s in own:
            s.stage(2)
        self.tr.exchange(SET_ACCUMULATOR_B, HALO)
        k2 = self._solve(1)
        self.tr.exchange(SET_SOLUTION, HALO)
        for s in own:
            s.finalize()
        self.tr.exchange(SET_STATE, HALO)
        self.last_products = (k1, k2)
        if device_cfl:
            dt = float(self._last_ctl[CG_DT])
            if self._last_ctl[CG_CFL_NONFINITE] != 0.0:
                self.status = "nonfinite"
        return dt, (k1, k2)

    def divb(self):
        """calculate_current_div_B (diagnostics.hpp:15-42) over the whole grid: (rms, max)."""
        rows = [s.divb_sums() for s in self.tr.own]
        (sq,) = self.tr.sum([[r[0]] for r in rows])
        mx = self.tr.max([max(r[1] for r in rows)])
        return math.sqrt(sq / (self.part.nx * self.part.ny)), mx


__all__ = ["Partition", "GpuSubdomain", "LocalTransport", "DistTransport", "DecomposedRun", "HALO",
           "MHDError", "DeviceCgGroup", "HostCgGroup"]
