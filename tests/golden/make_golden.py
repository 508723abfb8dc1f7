"""Writes tests/golden/step_hashes.json: SHA-256 of every section of three small worlds as the
scene builder makes them, and after the oracle steps them (the canonical step both the oracle
and the CUDA build compute bit for bit). The tests check the builder, the oracle and the CUDA
step against these, so a change to any of them that alters a result shows up as a mismatch.

    python tests/golden/make_golden.py

The reference's own step has no recorded outputs to pin against (its tests cover the scene
construction only); these are regression fixtures of this library's canonical form.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

CASES = {
    # name: (parameters, [batch sizes], FP64 solver sums)
    "bb_small": (dict(resolution=20, mesh_level=3, block_cap=4096, spray_cap=100000), [4, 4, 4, 4, 4, 4], True),
    "fixed_step_8cm": (dict(diameter=8, resolution=22, mesh_level=4, thickness=0.2, bullet=6, caliber=8, bullet_speed=300,
                            dt_max=2e-6, block_cap=4096, spray_cap=100000), [8, 8, 8], True),
    "fp32_sums": (dict(resolution=18, mesh_level=3, block_cap=4096, spray_cap=100000, bullet_speed=250), [4, 4, 4], False),
}


def section_hashes(world) -> dict:
    from natray_b200._abi import SECTIONS
    out = {name: hashlib.sha256(world.sec(name).tobytes()).hexdigest()[:32] for name in SECTIONS}
    out["STATE"] = hashlib.sha256(bytes(world.h.state)).hexdigest()[:32]
    return out


def main():
    from natray_b200 import Params, World, build_world
    from oracle.py import Oracle, set_threads
    set_threads(0)
    out = {}
    for name, (params, batches, fp64) in CASES.items():
        w0 = build_world(Params(**params))
        o = Oracle(w0.blob, fp64_dots=fp64)
        start = World(o.snapshot())  # after the measuring substep
        for n in batches:
            o.step(n)
        end = World(o.snapshot())
        out[name] = {"params": params, "batches": batches, "fp64_sums": fp64, "built": section_hashes(w0),
                     "start": section_hashes(start), "end": section_hashes(end), "end_state": end.state}
    (Path(__file__).parent / "step_hashes.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print("wrote", Path(__file__).parent / "step_hashes.json")


if __name__ == "__main__":
    main()
