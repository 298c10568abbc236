"""Test infrastructure only: ctypes bindings for the CPU oracle.

Two libraries live here, both built by ``oracle/Makefile``:

* ``liboracle.so``      -- the C restatement of the reference's IMEX step (``mhd_oracle.c``);
* ``_ref/libmhdref.so`` -- the reference's own headers (``include/*.hpp`` of
  RikibabManos/Magnetohydrodynamics_Simulator) compiled unmodified against the project-written
  Eigen subset, wrapped by ``ref_harness.cpp``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs may
import this module; the product never does. Fields are dense ``(ny, nx)`` float64 arrays in the
order rho, mx, my, E, bxf, byf (bxf on left faces, byf on bottom faces).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmhdref.so")
REF_SRC = os.environ.get("MHD_REFERENCE_DIR", "/root/reference")  # the reference sources (build only)

FIELDS = ("rho", "mx", "my", "E", "bxf", "byf")
PI_REF = 3.14159265359  # the reference driver's pi literal (src/integrator_main.cpp:36)

_dp = ctypes.POINTER(ctypes.c_double)


def build(with_reference: bool = True) -> None:
    """Compile the oracle (and the reference harness when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if with_reference and os.path.isdir(os.path.join(REF_SRC, "include")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("ct_abs_mode", ctypes.c_int),
        ("cg_tol", ctypes.c_double),
        ("cg_max_iters", ctypes.c_long),
    ]


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _ptr_array(fields):
    arr = (_dp * 6)()
    for k, f in enumerate(fields):
        arr[k] = _ptr(f)
    return arr


_oracle_lib = None


def oracle_lib():
    global _oracle_lib
    if _oracle_lib is None:
        if not os.path.exists(ORACLE_SO):
            build(with_reference=False)
        lib = ctypes.CDLL(ORACLE_SO)
        P = ctypes.POINTER(OrcParams)
        pa = ctypes.POINTER(_dp)
        lib.orc_explicit_rhs.argtypes = [P, pa, pa]
        lib.orc_imex_step.argtypes = [P, pa, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_long)]
        lib.orc_cfl_dt.argtypes = [P, pa, ctypes.c_double, ctypes.c_double]
        lib.orc_cfl_dt.restype = ctypes.c_double
        lib.orc_divb.argtypes = [P, _dp, _dp, _dp, _dp]
        lib.orc_snapshot.argtypes = [P, pa, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp]
        lib.orc_init_orszag_tang.argtypes = [P, pa]
        lib.orc_init_sine_wave.argtypes = [P, pa, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        lib.orc_cg_solve.argtypes = [P, ctypes.c_double, _dp, _dp, ctypes.POINTER(ctypes.c_long)]
        lib.orc_cg_solve.restype = ctypes.c_long
        lib.orc_corner_current_rhs.argtypes = [P, _dp, _dp, _dp]
        lib.orc_resistive_rate.argtypes = [P, _dp, _dp, ctypes.c_double, _dp, _dp]
        lib.orc_resistive_rate.restype = ctypes.c_long
        lib.orc_primitives.argtypes = [P, pa, _dp, _dp, _dp, _dp, _dp, _dp]
        _oracle_lib = lib
    return _oracle_lib


class Oracle:
    """The C restatement (dense periodic arrays)."""

    def __init__(self, nx, ny, dx, dy, eta, ct_abs_mode=0, cg_tol=0.0, cg_max_iters=0):
        self.lib = oracle_lib()
        self.p = OrcParams(nx, ny, dx, dy, eta, ct_abs_mode, cg_tol, cg_max_iters)
        self.nx, self.ny = nx, ny
        self.state = [np.zeros((ny, nx)) for _ in range(6)]

    # -- state
    def set_state(self, fields):
        self.state = [np.ascontiguousarray(f, dtype=np.float64).copy() for f in fields]

    def get_state(self):
        return [f.copy() for f in self.state]

    def init_orszag_tang(self):
        self.lib.orc_init_orszag_tang(ctypes.byref(self.p), _ptr_array(self.state))

    def init_sine_wave(self, az_amp=None, kx=0.0, ky=0.0, use_sin=False):
        if az_amp is None:  # reference amplitude 1/kx with kx = 2*pi/L
            kxx = kx if kx > 0 else 2 * PI_REF / (self.nx * self.p.dx)
            az_amp = 1.0 / kxx
        self.lib.orc_init_sine_wave(ctypes.byref(self.p), _ptr_array(self.state), az_amp, kx, ky, int(use_sin))

    # -- operators
    def explicit_rhs(self):
        out = [np.zeros((self.ny, self.nx)) for _ in range(6)]
        self.lib.orc_explicit_rhs(ctypes.byref(self.p), _ptr_array(self.state), _ptr_array(out))
        return out

    def primitives(self):
        out = [np.zeros((self.ny, self.nx)) for _ in range(6)]
        self.lib.orc_primitives(ctypes.byref(self.p), _ptr_array(self.state), *[_ptr(o) for o in out])
        return dict(zip(("rho", "vx", "vy", "p", "bxc", "byc"), out))

    def step(self, dt, alpha=None):
        if alpha is None:
            alpha = default_alpha(dt, self.p.eta)
        prods = (ctypes.c_long * 2)()
        self.lib.orc_imex_step(ctypes.byref(self.p), _ptr_array(self.state), dt, alpha, prods)
        return int(prods[0]), int(prods[1])

    def cfl_dt(self, courant=0.5, safety=0.9):
        return self.lib.orc_cfl_dt(ctypes.byref(self.p), _ptr_array(self.state), courant, safety)

    def divb(self):
        rms, mx = ctypes.c_double(), ctypes.c_double()
        self.lib.orc_divb(ctypes.byref(self.p), _ptr(self.state[4]), _ptr(self.state[5]),
                          ctypes.byref(rms), ctypes.byref(mx))
        return rms.value, mx.value

    def snapshot(self, ng=2, snapshot_rate=1, dt=0.0):
        """orc_snapshot: the snapshot file's doubles (header + 7 padded planes)."""
        out = np.zeros(9 + 7 * (self.p.nx + 2 * ng) * (self.p.ny + 2 * ng))
        self.lib.orc_snapshot(ctypes.byref(self.p), _ptr_array(self.state), ng, snapshot_rate, dt, _ptr(out))
        return out

    def cg_solve(self, alpha, rhs):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros_like(rhs)
        iters = ctypes.c_long()
        prods = self.lib.orc_cg_solve(ctypes.byref(self.p), alpha, _ptr(rhs), _ptr(x), ctypes.byref(iters))
        return x, int(prods)

    def corner_rhs(self):
        out = np.zeros((self.ny, self.nx))
        self.lib.orc_corner_current_rhs(ctypes.byref(self.p), _ptr(self.state[4]), _ptr(self.state[5]), _ptr(out))
        return out


def ars_gamma() -> float:
    """ARS(2,2,2) implicit diagonal (solvers.hpp:41)."""
    return (2.0 - np.sqrt(2.0)) / 2.0


def default_alpha(dt: float, eta: float) -> float:
    """The coefficient the reference driver builds its matrix with (integrator_main.cpp:89-90)."""
    return (dt * eta) * ars_gamma()


_ref_lib = None


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        lib = ctypes.CDLL(REF_SO)
        vp = ctypes.c_void_p
        lib.ref_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        lib.ref_create.restype = vp
        lib.ref_destroy.argtypes = [vp]
        lib.ref_init_orszag_tang.argtypes = [vp]
        lib.ref_init_dsw.argtypes = [vp]
        lib.ref_init_fixture.argtypes = [vp, ctypes.c_int]
        lib.ref_init_fixture.restype = ctypes.c_int
        lib.ref_set_state.argtypes = [vp] + [_dp] * 6
        lib.ref_get_state.argtypes = [vp] + [_dp] * 6
        lib.ref_get_primitives.argtypes = [vp] + [_dp] * 5
        lib.ref_cfl.argtypes = [vp]
        lib.ref_cfl.restype = ctypes.c_double
        lib.ref_set_alpha.argtypes = [vp, ctypes.c_double]
        lib.ref_step.argtypes = [vp, ctypes.c_double, ctypes.POINTER(ctypes.c_long)]
        lib.ref_divb.argtypes = [vp, _dp, _dp]
        lib.ref_write_snapshot.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        lib.ref_explicit_rhs.argtypes = [vp] + [_dp] * 6
        lib.ref_implicit_rate.argtypes = [vp, _dp, _dp, _dp]
        lib.ref_run.argtypes = [vp, ctypes.c_int, ctypes.c_double, _dp, _dp, ctypes.POINTER(ctypes.c_long)]
        _ref_lib = lib
    return _ref_lib


class Reference:
    """The reference's own IMEX step (compiled headers), driven through ref_harness.cpp."""

    def __init__(self, nx, ny, dx, dy, eta):
        self.lib = ref_lib()
        self.h = self.lib.ref_create(nx, ny, dx, dy, eta)
        self.nx, self.ny = nx, ny

    def __del__(self):
        try:
            self.lib.ref_destroy(self.h)
        except Exception:
            pass

    def init_orszag_tang(self):
        self.lib.ref_init_orszag_tang(self.h)

    def init_dsw(self):
        self.lib.ref_init_dsw(self.h)

    FIXTURES = ("alfven_wave", "gaussian_pulse", "acoustic_wave", "sausage", "kink")

    def init_fixture(self, name):
        """benchmarks.hpp:78-350, by name (FIXTURES)."""
        assert self.lib.ref_init_fixture(self.h, self.FIXTURES.index(name)) == 0

    def set_state(self, fields):
        fs = [np.ascontiguousarray(f, dtype=np.float64) for f in fields]
        self.lib.ref_set_state(self.h, *[_ptr(f) for f in fs])

    def get_state(self):
        out = [np.zeros((self.ny, self.nx)) for _ in range(6)]
        self.lib.ref_get_state(self.h, *[_ptr(o) for o in out])
        return out

    def primitives(self):
        out = [np.zeros((self.ny, self.nx)) for _ in range(5)]
        self.lib.ref_get_primitives(self.h, *[_ptr(o) for o in out])
        return dict(zip(("vx", "vy", "p", "bxc", "byc"), out))

    def cfl_dt(self):
        return self.lib.ref_cfl(self.h)

    def set_alpha(self, alpha):
        self.lib.ref_set_alpha(self.h, alpha)

    def step(self, dt):
        prods = (ctypes.c_long * 2)()
        self.lib.ref_step(self.h, dt, prods)
        return int(prods[0]), int(prods[1])

    def explicit_rhs(self):
        out = [np.zeros((self.ny, self.nx)) for _ in range(6)]
        self.lib.ref_explicit_rhs(self.h, *[_ptr(o) for o in out])
        return out

    def implicit_rate(self):
        bx = np.zeros((self.ny, self.nx))
        by = np.zeros((self.ny, self.nx))
        rhs = np.zeros((self.ny, self.nx))
        self.lib.ref_implicit_rate(self.h, _ptr(bx), _ptr(by), _ptr(rhs))
        return bx, by, rhs

    def divb(self):
        rms, mx = ctypes.c_double(), ctypes.c_double()
        self.lib.ref_divb(self.h, ctypes.byref(rms), ctypes.byref(mx))
        return rms.value, mx.value

    def write_snapshot(self, workdir, frame_index, snapshot_rate, dt):
        """integrator_main.cpp:107-109: the reference writes workdir/output/snapshot_NNNNNN.dat
        (its path is relative to the working directory); returns the file's bytes."""
        os.makedirs(os.path.join(workdir, "output"), exist_ok=True)
        cwd = os.getcwd()
        os.chdir(workdir)
        try:
            self.lib.ref_write_snapshot(self.h, frame_index, snapshot_rate, dt)
        finally:
            os.chdir(cwd)
        with open(os.path.join(workdir, "output", "snapshot_%06d.dat" % frame_index), "rb") as f:
            return f.read()

    def run(self, nsteps, dt_fixed=0.0, dts=None):
        """Driver loop of integrator_main.cpp:76-112; returns (dts, cg_products[nsteps, 2])."""
        dts_out = np.zeros(nsteps)
        prods = (ctypes.c_long * (2 * nsteps))()
        dts_in = None if dts is None else np.ascontiguousarray(dts, dtype=np.float64)
        self.lib.ref_run(self.h, nsteps, dt_fixed, None if dts_in is None else _ptr(dts_in), _ptr(dts_out), prods)
        return dts_out, np.array(prods[:], dtype=np.int64).reshape(nsteps, 2)


def rel_linf(a: np.ndarray, b: np.ndarray, floor: float = 0.0) -> float:
    """max|a-b| / max(max|b|, floor): per-field relative L-infinity error."""
    den = max(float(np.max(np.abs(b))), floor)
    if den == 0.0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b))) / den
