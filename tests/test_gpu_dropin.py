"""The drop-in, run: the reference's own driver program (src/integrator_main.cpp) built twice --
as the reference ships it, and switched to this library by the integration guide's diff
(include/mhd_b200_imex.hpp + `mhd_b200::` on its CFL, matrix, IMEX and snapshot calls) -- both by
oracle/Makefile's `dropin` target (oracle/dropin.py prints the two sources into the compiler).

Both programs run the Orszag-Tang vortex (choice 1 on stdin, benchmarks.hpp:419-452) on 64x64
with resistivity 1e-3, a dynamic CFL step and a snapshot every 5 steps up to t = 0.5, and write
output/snapshot_NNNNNN.dat in their working directories. Every file must exist in both runs and
agree: the header's grid, ghost width, rate and spacings exactly, its dt to 1e-12 relative, its
div B entries to 1e-12 absolute, and each of the 7 planes (ghosts included) to 1e-10 relative
L-infinity, the product's bar for multi-step runs.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from oracle.oracle import rel_linf

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "integrator_main_ref")
B200_BIN = os.path.join(ROOT, "oracle", "_ref", "integrator_main_b200")


def _run(binary, workdir):
    os.makedirs(os.path.join(workdir, "output"))
    r = subprocess.run([binary], input="1\n", capture_output=True, text=True, cwd=workdir, timeout=300)
    assert r.returncode == 0, (binary, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    assert "Simulation Finished!" in r.stdout, r.stdout[-2000:]
    files = sorted(os.listdir(os.path.join(workdir, "output")))
    return r.stdout, files


def _read(path):
    return np.fromfile(path, dtype=np.float64)


def test_reference_driver_runs_unchanged_on_the_gpu(tmp_path):
    import torch

    assert torch.cuda.is_available()
    for b in (REF_BIN, B200_BIN):
        assert os.path.exists(b), f"{b} was not built (make -C oracle dropin, with the reference sources)"
    out_ref, files_ref = _run(REF_BIN, str(tmp_path / "ref"))
    out_gpu, files_gpu = _run(B200_BIN, str(tmp_path / "b200"))
    assert files_ref == files_gpu and len(files_ref) >= 6, (files_ref, files_gpu)
    # the progress lines (percent of the run done at each snapshot) agree too
    prog = lambda s: [ln for ln in s.splitlines() if "% done" in ln]  # noqa: E731
    assert prog(out_ref) == prog(out_gpu)
    for name in files_ref:
        a = _read(str(tmp_path / "ref" / "output" / name))
        b = _read(str(tmp_path / "b200" / "output" / name))
        assert a.shape == b.shape, name
        ha, hb = a[:9], b[:9]
        assert np.array_equal(ha[:6], hb[:6]), (name, ha, hb)  # nx, ny, ng, rate, dx, dy
        assert abs(ha[6] - hb[6]) <= 1e-12 * abs(ha[6]), (name, ha[6], hb[6])  # dt
        assert abs(ha[7] - hb[7]) <= 1e-12 and abs(ha[8] - hb[8]) <= 1e-12, (name, ha[7:], hb[7:])
        nx, ny, ng = int(ha[0]), int(ha[1]), int(ha[2])
        planes_a = a[9:].reshape(7, ny + 2 * ng, nx + 2 * ng)
        planes_b = b[9:].reshape(7, ny + 2 * ng, nx + 2 * ng)
        for k, plane in enumerate(("rho", "E", "p", "vx", "vy", "bxc", "byc")):
            err = rel_linf(planes_b[k], planes_a[k])
            assert err <= 1e-10, (name, plane, err)
