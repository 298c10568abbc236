"""The CPU oracle under AddressSanitizer and UndefinedBehaviorSanitizer.

Every parity test trusts the oracle (oracle/mhd_oracle.c). `make -C oracle sanitize` builds a
driver of it with both sanitizers (oracle/sanitize_main.c), which runs each oracle entry point on
small grids with dx != dy (Orszag-Tang 36 x 28, four CFL steps; the decaying sine wave 32 x 20 in
the true-|v| corner mode with a capped solver) and stops with a report on any out-of-bounds
access, use after free, leak or undefined behaviour. Its results must also be the unsanitized
liboracle.so's, bit for bit (both build with strict IEEE arithmetic and no FMA contraction).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from oracle.oracle import Oracle, default_alpha


def test_oracle_runs_clean_under_sanitizers(tmp_path):
    b = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "sanitize"],
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if b.returncode != 0 and ("libsanitizer.spec" in b.stdout or "-lasan" in b.stdout):
        pytest.skip("no sanitizer runtime for the system compiler: " + b.stdout.strip()[-200:])
    assert b.returncode == 0, b.stdout
    out = tmp_path / "sanitized.bin"
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0:exitcode=23",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1:exitcode=24")
    r = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "oracle_sanitized"), str(out)], env=env,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-4000:]
    assert "runtime error" not in r.stdout and "AddressSanitizer" not in r.stdout, r.stdout[-4000:]
    got = np.fromfile(out, dtype=np.float64)

    # the same calls through the unsanitized library
    ot = Oracle(36, 28, 2 * np.pi / 36, 1.7 * np.pi / 28, 1e-2)
    ot.init_orszag_tang()
    for _ in range(4):
        dt = ot.cfl_dt(0.4, 0.9)
        ot.step(dt, alpha=default_alpha(dt, 1e-2))
    sw = Oracle(32, 20, 2 * np.pi / 32, 2 * np.pi / 20, 0.5, ct_abs_mode=1, cg_tol=1e-12, cg_max_iters=40)
    sw.init_sine_wave(az_amp=1e-3, kx=-1.0, ky=-1.0, use_sin=True)
    for _ in range(3):
        sw.step(1e-3, alpha=default_alpha(1e-3, 0.5))
    want = np.concatenate([np.stack(ot.get_state()).ravel(), np.stack(sw.get_state()).ravel(),
                           ot.snapshot(ng=2, snapshot_rate=5, dt=dt)])
    assert got.shape == want.shape
    assert np.array_equal(got, want)
