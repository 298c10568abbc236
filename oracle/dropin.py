"""Test infrastructure: the reference's own driver, src/integrator_main.cpp, prepared for the
drop-in check and printed to stdout (the Makefile pipes it straight into the compiler, so no copy
of the reference's source is written anywhere).

    python dropin.py REF_DIR ref    the driver as the reference ships it
    python dropin.py REF_DIR b200   the same driver switched to this library exactly as the
                                    integration guide's diff does: #include "mhd_b200_imex.hpp",
                                    `mhd_b200::` on CFL_condition_checker (:55, :80),
                                    generate_A_matrix (:59, :91) and IMEX (:99), the two
                                    matrix_solver.compute calls (:60, :92) dropped, and the
                                    snapshot block's fillGhostPeriodic + computePrimitives +
                                    write_data_to_binary_file (:107-109) replaced by
                                    mhd_b200::write_data_to_binary_file.

Both variants get the same values in the driver's "MAIN TWEAKABLE PROPERTIES" block
(integrator_main.cpp:25-30, the block the reference asks its users to edit): a 64x64 grid,
resistivity 1e-3 (so that every step runs the implicit solves), a snapshot every 5 steps and a
simulated duration of 0.5 (about thirty steps of Orszag-Tang, the last one clipped to end
exactly at 0.5). Every substitution must match the expected number of times, so a changed
reference fails loudly instead of producing another program.
"""
from __future__ import annotations

import os
import re
import sys

TWEAKS = [
    (r"const double animation_duration = [^;]*;", "const double animation_duration = 0.5;"),
    (r"const double resistivity = [^;]*;", "const double resistivity = 1e-3;"),
    (r"const int snapshot_frequency = [^;]*;", "const int snapshot_frequency = 5;"),
    (r"const int x_node_count = [^;]*;", "const int x_node_count = 64;"),
    (r"const int y_node_count = [^;]*;", "const int y_node_count = 64;"),
]

# (pattern, replacement, expected matches)
B200 = [
    (r'(#include "benchmarks\.hpp"\n)', r'\1#include "mhd_b200_imex.hpp"\n', 1),
    (r"(?<![\w:])CFL_condition_checker\(global_state\)", "mhd_b200::CFL_condition_checker(global_state)", 2),
    (r"(?<![\w:])generate_A_matrix\(global_state,", "mhd_b200::generate_A_matrix(global_state,", 2),
    (r"[ \t]*matrix_solver\.compute\(memory_storage\.A_matrix\);[ \t]*\n", "", 2),
    (r"(?<![\w:])IMEX\(global_state,", "mhd_b200::IMEX(global_state,", 1),
    (r"[ \t]*global_state\.fillGhostPeriodic\(\);[ \t]*\n"
     r"[ \t]*global_state\.computePrimitives\(\);[ \t]*\n"
     r"([ \t]*)write_data_to_binary_file\(global_state, frame_index, snapshot_frequency, current_time_step\);",
     r"\1mhd_b200::write_data_to_binary_file(global_state, frame_index, snapshot_frequency, current_time_step);", 1),
]


def _apply(src: str, pattern: str, repl: str, expected: int) -> str:
    out, n = re.subn(pattern, repl, src)
    if n != expected:
        raise SystemExit(f"dropin.py: pattern {pattern!r} matched {n} times, expected {expected}")
    return out


def driver_source(ref_dir: str, variant: str) -> str:
    with open(os.path.join(ref_dir, "src", "integrator_main.cpp")) as f:
        src = f.read()
    for pattern, repl in TWEAKS:
        src = _apply(src, pattern, repl, 1)
    if variant == "b200":
        for pattern, repl, expected in B200:
            src = _apply(src, pattern, repl, expected)
    elif variant != "ref":
        raise SystemExit(f"dropin.py: unknown variant {variant!r} (ref or b200)")
    return src


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit("usage: dropin.py REF_DIR ref|b200")
    sys.stdout.write(driver_source(sys.argv[1], sys.argv[2]))
