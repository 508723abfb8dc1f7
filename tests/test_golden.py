"""The committed fixtures of tests/golden/step_hashes.json (made by tests/golden/make_golden.py):
section hashes of three small worlds as built, after the measuring substep, and after the
oracle's batches of steps. The scene builder and the oracle must reproduce them (CPU), and the
CUDA step must reproduce the oracle's end state from the same start (GPU)."""
import json
from pathlib import Path

import pytest

from natray_b200 import Params, World, build_world

GOLDEN = json.loads((Path(__file__).parent / "golden" / "step_hashes.json").read_text())


def hashes(world):
    import sys
    sys.path.insert(0, str(Path(__file__).parent / "golden"))
    from make_golden import section_hashes
    return section_hashes(world)


def diff(a: dict, b: dict) -> list:
    return sorted(k for k in b if a.get(k) != b[k])


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_builder_and_oracle_reproduce_the_fixtures(name, oracle_threads):
    from oracle.py import Oracle
    g = GOLDEN[name]
    w0 = build_world(Params(**g["params"]))
    assert not diff(hashes(w0), g["built"]), f"{name}: scene builder"
    o = Oracle(w0.blob, fp64_dots=g["fp64_sums"])
    assert not diff(hashes(World(o.snapshot())), g["start"]), f"{name}: measuring substep"
    for n in g["batches"]:
        o.step(n)
    assert not diff(hashes(World(o.snapshot())), g["end"]), f"{name}: oracle steps"


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_cuda_step_reproduces_the_fixtures(name):
    from natray_b200.sim import Sim
    g = GOLDEN[name]
    w0 = build_world(Params(**g["params"]))
    s = Sim(world=w0, fp64_reductions=g["fp64_sums"])  # takes the measuring substep on the GPU
    assert not diff(hashes(s.snapshot()), g["start"]), f"{name}: measuring substep"
    for n in g["batches"]:
        assert s.step(n) == n
    d = diff(hashes(s.snapshot()), g["end"])
    assert not d, f"{name}: sections differ {d}"
