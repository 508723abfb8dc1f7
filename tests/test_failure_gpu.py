"""The failure path of the persistent pressure solve, exercised without faulting the GPU.

The solve runs as one cooperative launch whose CTAs meet at grid barriers (the reference runs its
iterations as host dispatches instead, fluid.wgsl:572-577, src/sim.rs:634-647). Every wait at a
barrier is bounded: after a limit of polls the CTA sets an error flag, returns, and the step
reports NTR_E_TIMEOUT. Here one CTA skips its first arrival (a flag nothing else sets) under a
short limit of 4096 polls: the step must fail promptly with NTR_E_TIMEOUT, the context must stay
usable, and a normal step from a restored snapshot must again equal the oracle bit for bit.
"""
import time

import pytest

from natray_b200 import World
from natray_b200._abi import NatrayError, check, lib
from natray_b200.sim import Sim
from oracle.py import Oracle

from test_parity_gpu import assert_worlds_equal, measured, small

pytestmark = pytest.mark.gpu

NTR_E_TIMEOUT = 5


def test_solver_barrier_timeout_is_reported_and_recoverable():
    w = measured(small())
    s = Sim(world=w)
    assert s.step(2) == 2
    saved = s.snapshot()
    check(lib().ntr_sim_test_barrier(s._h, 4096, 0))
    t0 = time.perf_counter()
    with pytest.raises(NatrayError) as e:
        s.step(1)
    assert e.value.status == NTR_E_TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    # Back to the default limit and no skipped arrival; the context still works.
    check(lib().ntr_sim_test_barrier(s._h, 0, 0xFFFFFFFF))
    s.restore(saved)
    o = Oracle(saved.blob)
    assert s.step(3) == o.step(3) == 3
    assert_worlds_equal(World(o.snapshot()), s.snapshot(), "after a solve whose barrier gave up")
    s.close()
