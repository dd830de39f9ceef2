"""The reference arm's rate counts the reference's own cell-updates.

The reference runs its time steps from t = 0, and the step at t = 0 updates
no field (the t > 0 guard of Source/Scheme/Scheme.inc.h:1032), so n time
steps are n - 1 updates per cell.  Runs the reference CPU build (built from
its sources under oracle/_ref) on the benchmark's 96^3 sample; skipped where
that binary has not been built.
"""
import math
import os

import pytest

import bench
from oracle.oracle import REF_BIN

pytestmark = pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference CPU build not built here")


def test_reference_sample_counts_updates_not_time_steps():
    r = bench.run_reference_sample(96, 3, procs=1)
    assert r["steps"] == 3 and r["updates"] == 2
    assert r["value"] > 0 and math.isfinite(r["value"])
    # the rate is the updates over the reference's own step-loop time
    assert r["value"] == pytest.approx(96 ** 3 * 2 / r["seconds"][0] / 1e9, rel=1e-12)


def test_reference_sample_refuses_a_single_time_step():
    with pytest.raises(ValueError, match="first time step"):
        bench.run_reference_sample(96, 1, procs=1)
