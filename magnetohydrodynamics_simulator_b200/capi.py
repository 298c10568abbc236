"""ctypes binding of the C ABI in include/mhd_b200.h (libmhd_b200.so, built in-tree).

This is the Python mirror of the drop-in boundary. There is no CPU fallback: if the library or an
sm_100 device is missing, every entry point raises MHDError.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmhd_b200.so")

MHD_OK = 0
STATUS_NAMES = {
    0: "MHD_OK",
    1: "MHD_ERR_INVALID_ARGUMENT",
    2: "MHD_ERR_CUDA",
    3: "MHD_ERR_NONFINITE",
    4: "MHD_ERR_CG_NOT_CONVERGED",
    5: "MHD_ERR_TIMEOUT",
    6: "MHD_ERR_NO_DEVICE",
    7: "MHD_ERR_OUT_OF_MEMORY",
    8: "MHD_ERR_NO_STATE",
    9: "MHD_ERR_TOO_LARGE",
    10: "MHD_ERR_IO",
}
LAYOUT_DENSE = 0
LAYOUT_PADDED = 1
CT_REFERENCE = 0
CT_TRUE_ABS = 1
FIELDS = ("rho", "mx", "my", "E", "bxf", "byf")
PRIMITIVES = ("rho", "vx", "vy", "p", "bxc", "byc")


class MHDError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}")


class Params(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int),
        ("ny", ctypes.c_int),
        ("dx", ctypes.c_double),
        ("dy", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("ct_mode", ctypes.c_int),
        ("cg_tol", ctypes.c_double),
        ("cg_max_iters", ctypes.c_longlong),
        ("courant", ctypes.c_double),
        ("safety", ctypes.c_double),
        ("cg_timeout_s", ctypes.c_double),
    ]


class BatchTuning(ctypes.Structure):
    _fields_ = [
        ("stage_rows", ctypes.c_int),
        ("cg_rows", ctypes.c_int),
        ("cg_order", ctypes.c_int),
        ("stage_tail_rows", ctypes.c_int),
        ("stage_ms", ctypes.c_double),
        ("cg_ms", ctypes.c_double),
    ]


_dp = ctypes.POINTER(ctypes.c_double)
_lib = None


def load_library() -> ctypes.CDLL:
    """Load libmhd_b200.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MHDError(6, f"{LIB_PATH} is missing (run __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    P6 = _dp * 6
    lib.mhd_default_params.argtypes = [ctypes.POINTER(Params), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.mhd_create.argtypes = [ctypes.POINTER(Params), vp, ctypes.POINTER(vp)]
    lib.mhd_destroy.argtypes = [vp]
    lib.mhd_set_state.argtypes = [vp, P6, ctypes.c_int, ctypes.c_int]
    lib.mhd_get_state.argtypes = [vp, P6, ctypes.c_int, ctypes.c_int]
    lib.mhd_set_state_async.argtypes = [vp, P6]
    lib.mhd_get_state_async.argtypes = [vp, P6]
    lib.mhd_transfers_wait.argtypes = [vp]
    lib.mhd_set_state_device.argtypes = [vp, P6]
    lib.mhd_get_state_device.argtypes = [vp, P6]
    lib.mhd_get_primitives.argtypes = [vp, P6, ctypes.c_int, ctypes.c_int]
    lib.mhd_set_implicit_coefficient.argtypes = [vp, ctypes.c_double]
    lib.mhd_step.argtypes = [vp, ctypes.c_double]
    lib.mhd_run.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp,
                            ctypes.POINTER(ctypes.c_longlong)]
    lib.mhd_resistive_rate.argtypes = [vp, ctypes.c_int, ctypes.c_double, vp, vp, vp, vp,
                                       ctypes.POINTER(ctypes.c_longlong)]
    lib.mhd_set_kernel_timing.argtypes = [vp, ctypes.c_int]
    lib.mhd_kernel_times.argtypes = [vp, _dp, ctypes.POINTER(ctypes.c_longlong)]
    lib.mhd_cfl_dt.argtypes = [vp, _dp]
    lib.mhd_divb.argtypes = [vp, _dp, _dp]
    lib.mhd_snapshot_bytes.argtypes = [vp, ctypes.c_int]
    lib.mhd_snapshot_bytes.restype = ctypes.c_size_t
    lib.mhd_snapshot_write.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    lib.mhd_snapshot_wait.argtypes = [vp]
    lib.mhd_snapshot_pack.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, vp]
    lib.mhd_synchronize.argtypes = [vp]
    lib.mhd_last_cg_products.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.mhd_cg_products_sum.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.mhd_state_device_pointers.argtypes = [vp, P6]
    lib.mhd_stream.argtypes = [vp]
    lib.mhd_stream.restype = vp
    lib.mhd_launches_per_step.argtypes = [vp]
    lib.mhd_status_string.argtypes = [ctypes.c_int]
    lib.mhd_status_string.restype = ctypes.c_char_p
    lib.mhd_device_available.argtypes = []
    ip = ctypes.POINTER(ctypes.c_int)
    llp = ctypes.POINTER(ctypes.c_longlong)
    tp = ctypes.POINTER(BatchTuning)
    lib.mhd_batch_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int, vp, ctypes.POINTER(vp)]
    lib.mhd_batch_destroy.argtypes = [vp]
    lib.mhd_batch_count.argtypes = [vp]
    lib.mhd_batch_set_state.argtypes = [vp, ctypes.c_int, P6]
    lib.mhd_batch_get_state.argtypes = [vp, ctypes.c_int, P6]
    lib.mhd_batch_set_state_device.argtypes = [vp, ctypes.c_int, P6]
    lib.mhd_batch_get_state_device.argtypes = [vp, ctypes.c_int, P6]
    lib.mhd_batch_set_implicit_coefficient.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    lib.mhd_batch_step.argtypes = [vp, _dp]
    lib.mhd_batch_run.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, llp]
    lib.mhd_batch_autotune.argtypes = [vp, tp]
    lib.mhd_batch_set_tuning.argtypes = [vp, tp]
    lib.mhd_batch_get_tuning.argtypes = [vp, tp]
    lib.mhd_batch_synchronize.argtypes = [vp, ip]
    lib.mhd_batch_last_cg_products.argtypes = [vp, llp]
    lib.mhd_batch_cfl_dt.argtypes = [vp, ctypes.c_int, _dp]
    lib.mhd_batch_divb.argtypes = [vp, ctypes.c_int, _dp, _dp]
    lib.mhd_batch_stream.argtypes = [vp]
    lib.mhd_batch_stream.restype = vp
    lib.mhd_batch_launches_per_step.argtypes = [vp]
    lib.mhd_resistive_rate_noalloc.argtypes = [ctypes.POINTER(Params), ctypes.c_int, ctypes.c_double,
                                               vp, vp, vp, vp, llp, vp]
    lib.mhd_adj_create.argtypes = [ctypes.POINTER(Params), ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                   vp, ctypes.POINTER(vp)]
    lib.mhd_adj_create_ex.argtypes = [ctypes.POINTER(Params), ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, vp, ctypes.POINTER(vp)]
    lib.mhd_adj_device_bytes.argtypes = [vp]
    lib.mhd_adj_device_bytes.restype = ctypes.c_size_t
    lib.mhd_adj_destroy.argtypes = [vp]
    lib.mhd_adj_set_eta.argtypes = [vp, ctypes.c_double]
    lib.mhd_adj_forward.argtypes = [vp, P6, P6]
    lib.mhd_adj_backward.argtypes = [vp, P6, P6, _dp]
    lib.mhd_adj_step_vjp.argtypes = [vp, P6, P6, P6, _dp]
    lib.mhd_adj_rate_vjp.argtypes = [vp, P6, P6, P6]
    lib.mhd_adj_launch_counts.argtypes = [vp, ip, ip]
    lib.mhd_adj_stream.argtypes = [vp]
    lib.mhd_adj_stream.restype = vp
    _lib = lib
    return lib


def _check(status: int, where: str) -> None:
    if status != MHD_OK:
        raise MHDError(status, where)


def _host_ptrs(arrays: Sequence[np.ndarray]):
    arr = (_dp * 6)()
    for k, a in enumerate(arrays):
        if a is None:
            arr[k] = None
        else:
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("fields must be C-contiguous float64 arrays")
            arr[k] = a.ctypes.data_as(_dp)
    return arr


def _device_ptrs(ptrs: Sequence[int]):
    arr = (_dp * 6)()
    for k, p in enumerate(ptrs):
        arr[k] = ctypes.cast(ctypes.c_void_p(int(p)), _dp) if p else None
    return arr


def device_available() -> bool:
    return bool(load_library().mhd_device_available())


class Context:
    """One simulation on the GPU: the device-resident counterpart of the reference's Grid +
    integrator_reserved_memory + solver objects (src/integrator_main.cpp:34-48)."""

    def __init__(self, nx: int, ny: int, dx: float, dy: float, eta: float, *, ct_mode: int = 0,
                 cg_tol: float = 0.0, cg_max_iters: int = 0, courant: float = 0.5,
                 safety: float = 0.9, cg_timeout_s: float = 30.0, stream: int | None = None):
        self.lib = load_library()
        self.nx, self.ny = int(nx), int(ny)
        p = Params()
        _check(self.lib.mhd_default_params(ctypes.byref(p), nx, ny, dx, dy, eta), "mhd_default_params")
        p.ct_mode = ct_mode
        p.cg_tol = cg_tol
        p.cg_max_iters = cg_max_iters
        p.courant = courant
        p.safety = safety
        p.cg_timeout_s = cg_timeout_s
        self.params = p
        h = ctypes.c_void_p()
        _check(self.lib.mhd_create(ctypes.byref(p), ctypes.c_void_p(stream) if stream else None,
                                   ctypes.byref(h)), "mhd_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- state
    def _shape(self, layout, ng):
        if layout == LAYOUT_DENSE:
            return (self.ny, self.nx)
        return (self.ny + 2 * ng, self.nx + 2 * ng)

    def set_state(self, fields: Sequence[np.ndarray], layout: int = LAYOUT_DENSE, ng: int = 2):
        fs = [np.ascontiguousarray(f, dtype=np.float64) for f in fields]
        for f in fs:
            if f.shape != self._shape(layout, ng):
                raise ValueError(f"field shape {f.shape} != {self._shape(layout, ng)}")
        _check(self.lib.mhd_set_state(self.h, _host_ptrs(fs), layout, ng), "mhd_set_state")

    def get_state(self, layout: int = LAYOUT_DENSE, ng: int = 2):
        out = [np.empty(self._shape(layout, ng)) for _ in range(6)]
        _check(self.lib.mhd_get_state(self.h, _host_ptrs(out), layout, ng), "mhd_get_state")
        return out

    def get_state_into(self, out: Sequence[np.ndarray], layout: int = LAYOUT_DENSE, ng: int = 2):
        _check(self.lib.mhd_get_state(self.h, _host_ptrs(out), layout, ng), "mhd_get_state")

    def set_state_async(self, fields: Sequence[np.ndarray]):
        """Pipelined upload of dense host planes (pinned for overlap); see mhd_set_state_async.
        The arrays must stay alive and untouched until transfers_wait()."""
        _check(self.lib.mhd_set_state_async(self.h, _host_ptrs(fields)), "mhd_set_state_async")

    def get_state_async(self, out: Sequence[np.ndarray]):
        """Pipelined read-back into dense host planes; ready after transfers_wait()."""
        _check(self.lib.mhd_get_state_async(self.h, _host_ptrs(out)), "mhd_get_state_async")

    def transfers_wait(self):
        _check(self.lib.mhd_transfers_wait(self.h), "mhd_transfers_wait")

    def set_state_device(self, ptrs: Sequence[int]):
        _check(self.lib.mhd_set_state_device(self.h, _device_ptrs(ptrs)), "mhd_set_state_device")

    def get_state_device(self, ptrs: Sequence[int]):
        _check(self.lib.mhd_get_state_device(self.h, _device_ptrs(ptrs)), "mhd_get_state_device")

    def state_device_pointers(self):
        arr = (_dp * 6)()
        _check(self.lib.mhd_state_device_pointers(self.h, arr), "mhd_state_device_pointers")
        return [ctypes.cast(arr[k], ctypes.c_void_p).value for k in range(6)]

    def primitives(self, layout: int = LAYOUT_DENSE, ng: int = 2):
        out = [np.empty(self._shape(layout, ng)) for _ in range(6)]
        _check(self.lib.mhd_get_primitives(self.h, _host_ptrs(out), layout, ng), "mhd_get_primitives")
        return dict(zip(PRIMITIVES, out))

    # ---------------------------------------------------------------- stepping
    def set_implicit_coefficient(self, alpha: float):
        _check(self.lib.mhd_set_implicit_coefficient(self.h, alpha), "mhd_set_implicit_coefficient")

    def step(self, dt: float):
        _check(self.lib.mhd_step(self.h, dt), "mhd_step")

    def run(self, nsteps: int, dt_fixed: float = 0.0, t_end: float = 0.0, record: bool = True):
        dts = np.zeros(nsteps) if record else None
        prods = np.zeros((nsteps, 2), dtype=np.int64) if record else None
        _check(self.lib.mhd_run(self.h, nsteps, dt_fixed, t_end,
                                dts.ctypes.data_as(_dp) if record else None,
                                prods.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)) if record else None),
               "mhd_run")
        return dts, prods

    def synchronize(self):
        _check(self.lib.mhd_synchronize(self.h), "mhd_synchronize")

    def synchronize_status(self) -> int:
        return int(self.lib.mhd_synchronize(self.h))

    def last_cg_products(self):
        out = (ctypes.c_longlong * 2)()
        _check(self.lib.mhd_last_cg_products(self.h, out), "mhd_last_cg_products")
        return int(out[0]), int(out[1])

    def cg_products_sum(self):
        """Products of the first and of the second solve of every step so far, summed."""
        out = (ctypes.c_longlong * 2)()
        _check(self.lib.mhd_cg_products_sum(self.h, out), "mhd_cg_products_sum")
        return int(out[0]), int(out[1])

    def resistive_rate(self, bxf: int, byf: int, bx_rate: int, by_rate: int, *,
                       solve_implicitly: bool, alpha: float = 0.0) -> int:
        """resistive_B_term (solvers.hpp:445-489) on device planes given by their addresses;
        returns the implicit solve's matrix-vector products."""
        prods = ctypes.c_longlong()
        _check(self.lib.mhd_resistive_rate(self.h, int(solve_implicitly), alpha, ctypes.c_void_p(bxf),
                                           ctypes.c_void_p(byf), ctypes.c_void_p(bx_rate),
                                           ctypes.c_void_p(by_rate), ctypes.byref(prods)),
               "mhd_resistive_rate")
        return int(prods.value)

    def cfl_dt(self) -> float:
        v = ctypes.c_double()
        _check(self.lib.mhd_cfl_dt(self.h, ctypes.byref(v)), "mhd_cfl_dt")
        return v.value

    def divb(self):
        rms, mx = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.mhd_divb(self.h, ctypes.byref(rms), ctypes.byref(mx)), "mhd_divb")
        return rms.value, mx.value

    # -- snapshots in the reference's file format (diagnostics.hpp:90-131)
    def snapshot_bytes(self, ng: int = 2) -> int:
        return int(self.lib.mhd_snapshot_bytes(self.h, ng))

    def snapshot_write(self, path: str, ng: int = 2, snapshot_rate: int = 1, dt: float = 0.0):
        """Write the current state's snapshot file asynchronously (see mhd_snapshot_write)."""
        _check(self.lib.mhd_snapshot_write(self.h, os.fsencode(path), ng, snapshot_rate, dt),
               "mhd_snapshot_write")

    def snapshot_wait(self):
        _check(self.lib.mhd_snapshot_wait(self.h), "mhd_snapshot_wait")

    def snapshot_pack(self, ng: int = 2, snapshot_rate: int = 1, dt: float = 0.0) -> np.ndarray:
        """The snapshot file's doubles (9-double header, then 7 padded planes)."""
        n = self.snapshot_bytes(ng)
        if n == 0:
            raise MHDError(1, "snapshot_pack: invalid ng")
        out = np.empty(n // 8, dtype=np.float64)
        _check(self.lib.mhd_snapshot_pack(self.h, ng, snapshot_rate, dt, out.ctypes.data),
               "mhd_snapshot_pack")
        return out

    @property
    def stream(self) -> int:
        return self.lib.mhd_stream(self.h) or 0

    @property
    def launches_per_step(self) -> int:
        return int(self.lib.mhd_launches_per_step(self.h))


_TUNING_KEYS = ("stage_rows", "cg_rows", "cg_order", "stage_tail_rows", "stage_ms", "cg_ms")


class Batch:
    """Many independent periodic simulations of uneven sizes stepped together (one launch per
    stage for the whole batch). Each instance is specified like a Context: a dict with keys
    nx, ny, dx, dy, eta and optionally ct_mode, cg_tol, cg_max_iters, courant, safety,
    cg_timeout_s."""

    def __init__(self, instances: Sequence[dict], stream: int | None = None):
        self.lib = load_library()
        n = len(instances)
        arr = (Params * n)()
        self.shapes = []
        for k, spec in enumerate(instances):
            p = arr[k]
            _check(self.lib.mhd_default_params(ctypes.byref(p), int(spec["nx"]), int(spec["ny"]),
                                               float(spec["dx"]), float(spec["dy"]),
                                               float(spec["eta"])), "mhd_default_params")
            for key in ("ct_mode", "cg_tol", "cg_max_iters", "courant", "safety", "cg_timeout_s"):
                if key in spec:
                    setattr(p, key, spec[key])
            self.shapes.append((int(spec["ny"]), int(spec["nx"])))
        self.params = arr
        h = ctypes.c_void_p()
        _check(self.lib.mhd_batch_create(arr, n, ctypes.c_void_p(stream) if stream else None,
                                         ctypes.byref(h)), "mhd_batch_create")
        self.h = h
        self.count = n

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return self.count

    def set_state(self, index: int, fields: Sequence[np.ndarray]):
        fs = [np.ascontiguousarray(f, dtype=np.float64) for f in fields]
        for f in fs:
            if f.shape != self.shapes[index]:
                raise ValueError(f"field shape {f.shape} != {self.shapes[index]}")
        _check(self.lib.mhd_batch_set_state(self.h, index, _host_ptrs(fs)), "mhd_batch_set_state")

    def get_state(self, index: int):
        out = [np.empty(self.shapes[index]) for _ in range(6)]
        _check(self.lib.mhd_batch_get_state(self.h, index, _host_ptrs(out)), "mhd_batch_get_state")
        return out

    def get_state_into(self, index: int, out: Sequence[np.ndarray]):
        _check(self.lib.mhd_batch_get_state(self.h, index, _host_ptrs(out)), "mhd_batch_get_state")

    def set_state_device(self, index: int, ptrs: Sequence[int]):
        _check(self.lib.mhd_batch_set_state_device(self.h, index, _device_ptrs(ptrs)),
               "mhd_batch_set_state_device")

    def get_state_device(self, index: int, ptrs: Sequence[int]):
        _check(self.lib.mhd_batch_get_state_device(self.h, index, _device_ptrs(ptrs)),
               "mhd_batch_get_state_device")

    def set_implicit_coefficient(self, index: int, alpha: float):
        _check(self.lib.mhd_batch_set_implicit_coefficient(self.h, index, alpha),
               "mhd_batch_set_implicit_coefficient")

    def step(self, dts: Sequence[float] | None = None):
        if dts is None:
            _check(self.lib.mhd_batch_step(self.h, None), "mhd_batch_step")
            return
        d = np.ascontiguousarray(dts, dtype=np.float64)
        if d.shape != (self.count,):
            raise ValueError("dts must hold one dt per instance")
        _check(self.lib.mhd_batch_step(self.h, d.ctypes.data_as(_dp)), "mhd_batch_step")

    def run(self, nsteps: int, dt_fixed: float = 0.0, t_end: float = 0.0, record: bool = True):
        """Returns dts[count, nsteps] and cg_products[count, nsteps, 2] (None, None unless
        record)."""
        dts = np.zeros((self.count, nsteps)) if record else None
        prods = np.zeros((self.count, nsteps, 2), dtype=np.int64) if record else None
        _check(self.lib.mhd_batch_run(
            self.h, nsteps, dt_fixed, t_end, dts.ctypes.data_as(_dp) if record else None,
            prods.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)) if record else None),
            "mhd_batch_run")
        return dts, prods

    def autotune(self) -> dict:
        t = BatchTuning()
        _check(self.lib.mhd_batch_autotune(self.h, ctypes.byref(t)), "mhd_batch_autotune")
        return {k: getattr(t, k) for k in _TUNING_KEYS}

    def tuning(self) -> dict:
        t = BatchTuning()
        _check(self.lib.mhd_batch_get_tuning(self.h, ctypes.byref(t)), "mhd_batch_get_tuning")
        return {k: getattr(t, k) for k in _TUNING_KEYS}

    def set_tuning(self, stage_rows: int, cg_rows: int, cg_order: int = 0, stage_tail_rows: int = 0):
        t = BatchTuning(stage_rows, cg_rows, cg_order, stage_tail_rows, 0.0, 0.0)
        _check(self.lib.mhd_batch_set_tuning(self.h, ctypes.byref(t)), "mhd_batch_set_tuning")

    def synchronize_status(self):
        """(worst status, per-instance statuses); clears the device statuses."""
        per = (ctypes.c_int * self.count)()
        worst = int(self.lib.mhd_batch_synchronize(self.h, per))
        return worst, [int(v) for v in per]

    def synchronize(self):
        worst, _ = self.synchronize_status()
        _check(worst, "mhd_batch_synchronize")

    def last_cg_products(self) -> np.ndarray:
        out = np.zeros((self.count, 2), dtype=np.int64)
        _check(self.lib.mhd_batch_last_cg_products(
            self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))), "mhd_batch_last_cg_products")
        return out

    def cfl_dt(self, index: int) -> float:
        v = ctypes.c_double()
        _check(self.lib.mhd_batch_cfl_dt(self.h, index, ctypes.byref(v)), "mhd_batch_cfl_dt")
        return v.value

    def divb(self, index: int):
        rms, mx = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.mhd_batch_divb(self.h, index, ctypes.byref(rms), ctypes.byref(mx)),
               "mhd_batch_divb")
        return rms.value, mx.value

    @property
    def stream(self) -> int:
        return self.lib.mhd_batch_stream(self.h) or 0

    @property
    def launches_per_step(self) -> int:
        return int(self.lib.mhd_batch_launches_per_step(self.h))


class Adjoint:
    """Differentiable fixed-dt trajectory of `nsteps` IMEX steps of one grid (the mhd_adj_* ABI):
    forward keeps every `checkpoint_every`-th state, backward recomputes each segment and runs the
    hand-written adjoint steps. recompute_solves: keep one segment's implicit solutions instead of
    every step's and re-solve in the backward pass (memory O(nsteps/k + k) planes). State arguments are lists of six device addresses (dense planes
    rho, mx, my, E, bxf, byf). Calls are synchronous on the object's own stream."""

    def __init__(self, nx: int, ny: int, dx: float, dy: float, eta: float, dt: float, nsteps: int,
                 checkpoint_every: int = 10, *, ct_mode: int = 0, cg_tol: float = 0.0,
                 cg_max_iters: int = 0, cg_timeout_s: float = 30.0, stream: int | None = None,
                 recompute_solves: bool = False):
        self.lib = load_library()
        self.nx, self.ny, self.dt, self.nsteps = int(nx), int(ny), float(dt), int(nsteps)
        self.checkpoint_every = int(checkpoint_every)
        p = Params()
        _check(self.lib.mhd_default_params(ctypes.byref(p), nx, ny, dx, dy, eta), "mhd_default_params")
        p.ct_mode = ct_mode
        p.cg_tol = cg_tol
        p.cg_max_iters = cg_max_iters
        p.cg_timeout_s = cg_timeout_s
        self.params = p
        self.eta = float(eta)
        h = ctypes.c_void_p()
        _check(self.lib.mhd_adj_create_ex(ctypes.byref(p), dt, nsteps, checkpoint_every,
                                          1 if recompute_solves else 0,
                                          ctypes.c_void_p(stream) if stream else None, ctypes.byref(h)),
               "mhd_adj_create_ex")
        self.h = h

    @property
    def device_bytes(self) -> int:
        """Device memory of the object's planes (checkpoints, segment slots, solutions, scratch)."""
        return int(self.lib.mhd_adj_device_bytes(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_adj_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_eta(self, eta: float):
        _check(self.lib.mhd_adj_set_eta(self.h, float(eta)), "mhd_adj_set_eta")
        self.eta = float(eta)

    def forward(self, u0: Sequence[int], uT: Sequence[int]):
        _check(self.lib.mhd_adj_forward(self.h, _device_ptrs(u0), _device_ptrs(uT)), "mhd_adj_forward")

    def backward(self, grad_uT: Sequence[int], grad_u0: Sequence[int]) -> float:
        g = ctypes.c_double()
        _check(self.lib.mhd_adj_backward(self.h, _device_ptrs(grad_uT), _device_ptrs(grad_u0),
                                         ctypes.byref(g)), "mhd_adj_backward")
        return g.value

    def step_vjp(self, u: Sequence[int], lam_next: Sequence[int], lam: Sequence[int]) -> float:
        g = ctypes.c_double()
        _check(self.lib.mhd_adj_step_vjp(self.h, _device_ptrs(u), _device_ptrs(lam_next),
                                         _device_ptrs(lam), ctypes.byref(g)), "mhd_adj_step_vjp")
        return g.value

    def rate_vjp(self, u: Sequence[int], w: Sequence[int], out: Sequence[int]):
        _check(self.lib.mhd_adj_rate_vjp(self.h, _device_ptrs(u), _device_ptrs(w), _device_ptrs(out)),
               "mhd_adj_rate_vjp")

    @property
    def stream(self) -> int:
        return self.lib.mhd_adj_stream(self.h) or 0

    def launch_counts(self):
        f, a = ctypes.c_int(), ctypes.c_int()
        _check(self.lib.mhd_adj_launch_counts(self.h, ctypes.byref(f), ctypes.byref(a)),
               "mhd_adj_launch_counts")
        return int(f.value), int(a.value)


def ars_gamma() -> float:
    """ARS(2,2,2) implicit diagonal g = 1 - 1/sqrt(2) (solvers.hpp:41)."""
    return (2.0 - np.sqrt(2.0)) / 2.0
