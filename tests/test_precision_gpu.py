"""The precision study of the 1M-particle scene (976,915 particles, a level-6 membrane, an 8 mm
sphere at 350 m/s): the product (FP32 state and grid arithmetic, FP64 solver sums, on the GPU)
against the oracle with every real in FP64, from the same start, relative L2 errors of positions,
velocities, particle pressure, membrane positions and the membrane's major principal stretch.

The bounds are the measured errors (tests/precision_study.py, 1000 steps at solver tolerances
1e-5 and 1e-7 alike) with a margin of three to five:

- before the sphere reaches the membrane (step 70), and in the same scene with the sphere at
  1 m/s (it never arrives): positions within 2e-7 (measured 5e-8), membrane positions within
  3e-6 (6e-7), velocities and pressure within 3e-3 (8e-4 and 6e-4: the same at the tight
  tolerance, so FP32 rounding and not the solver's stopping point), stretch within 1e-3 (2e-4);
- after it the membrane tears at different substeps and triangles on the two sides, a discrete
  event (12 torn triangles against 13 at step 80), and the velocity and pressure fields differ
  where it does (0.33 and 0.43 at step 80, 0.14 and 0.06 at step 100); positions stay within
  1e-4 (1.4e-5 at step 100), membrane positions within 5e-4 (5e-5), stretch within 3e-2 (4.5e-3)
  and the torn counts within a quarter of each other.

Run with -s to see the tables."""
import pytest

from precision_study import study

pytestmark = pytest.mark.gpu


def test_fp32_product_tracks_fp64_through_the_impact(oracle_threads):
    rows = study(124, 100, 20, 1e-5)
    for r in rows:
        if r["step"] <= 60:
            assert r["torn"] == [0, 0]
            assert r["x"] < 2e-7 and r["mem_x"] < 3e-6, r
            assert r["v"] < 3e-3 and r["p"] < 3e-3 and r["stretch"] < 1e-3, r
        else:
            assert r["x"] < 1e-4 and r["mem_x"] < 5e-4 and r["stretch"] < 3e-2, r
            a, b = r["torn"]
            assert abs(a - b) <= max(3, 0.25 * max(a, b)), r
    assert rows[-1]["torn"][0] > 0  # the step range covers the impact


def test_fp32_product_tracks_fp64_at_rest(oracle_threads):
    rows = study(124, 200, 100, 1e-5, speed=1.0)
    for r in rows:
        assert r["torn"] == [0, 0]
        assert r["x"] < 1e-6 and r["mem_x"] < 1e-5, r
        assert r["v"] < 3e-3 and r["p"] < 5e-3 and r["stretch"] < 1e-3, r
