"""The bench's roofline accounting, on the CPU: the algorithmic bytes of a launch of each kernel
that can lead the step's profile, the step-level bytes from the device's work counters, and the
DRAM traffic lines the bench reads from the committed ncu summaries."""
import importlib.util
import sys
from pathlib import Path
from types import SimpleNamespace

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bench_under_test"] = mod
    spec.loader.exec_module(mod)
    return mod


def test_kernel_bytes_per_launch():
    b = _bench()
    st = {"n_blocks": 3000, "_n_water": 100_000}
    cells = 3000 * 64
    # P2G: 80 B of particle and its 4 B index read, each cell's 4 B particle count written.
    assert b.algorithmic_bytes("k_p2g", st, 1_000_000, 10) == 84.0 * 1_000_000 + 4.0 * cells
    # The solve: 48 B per water cell and iteration, 40 B per water cell to set up.
    assert b.algorithmic_bytes("k_solve<true>", st, 1_000_000, 10) == 48.0 * 100_000 * 10 + 40.0 * 100_000
    # At least one iteration is counted (a solve that stops at once still sets up and checks).
    assert b.algorithmic_bytes("k_solve<false>", st, 1_000_000, 0) == 48.0 * 100_000 + 40.0 * 100_000
    # G2P: the particle read and written (80 + 80 B) and its index, the cells' 8 fields once.
    assert b.algorithmic_bytes("k_g2p<128>", st, 1_000_000, 10) == 164.0 * 1_000_000 + 32.0 * cells
    # Other kernels carry no per-launch figure.
    assert b.algorithmic_bytes("k_mark", st, 1_000_000, 10) == 0.0


def test_step_bytes_from_work_counters():
    from natray_b200.sim import Sim
    fake = SimpleNamespace(info=SimpleNamespace(n_particles=1000, n_verts=50, n_tris=96))
    work = {"steps": 3, "cells": 640, "water_iters": 2000, "mem_substeps": 6, "gas_substeps": 700, "spray": 10}
    want = (160.0 * 1000 * 3 + 160.0 * 640 + 48.0 * 2000 + (256.0 * 50 + 32.0 * 96) * 6 + 44.0 * 700 + 48.0 * 10)
    assert Sim.algorithmic_bytes(fake, work) == want


@pytest.mark.parametrize("kernel", ["k_p2g", "k_solve", "k_g2p"])
def test_traffic_lines_the_bench_reads(kernel):
    # The bench takes `traffic` for the leading kernel from profiles/<kernel>.md: each kernel that
    # can lead has one such line, a byte count of one launch, below the kernel's summary command.
    text = (ROOT / "profiles" / f"{kernel}.md").read_text()
    lines = [ln for ln in text.splitlines() if ln.startswith("traffic_per_launch_bytes:")]
    assert len(lines) == 1
    value = float(lines[0].split(":", 1)[1])
    assert 1e6 < value < 1e9
    assert "ncu " in text and "--clock-control none" in text
