"""Arrival times and maximum elevation (okl/Analysis/*) on the engine (GPU).

With CalcArrivalTimes / CalcMaximumElevation set at initDeviceVariables the
engine updates both per-node arrays after every time step, inside its
captured step graph.  They must equal, bit for bit, the arrays of the
reference program itself (tests/golden/walls_analysis_N3.npz) and the
oracle's on a curved lake run by a step count, and they are reported only
when enabled.
"""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.deviceclass import E_ARG, EsdgError, Solver
from oracle.oracle import OracleProblem
from tests.golden import fixtures

pytestmark = pytest.mark.gpu


def test_engine_analysis_matches_reference_bitwise():
    prob, q_ref, z = fixtures.load("walls_analysis_N3")
    s = Solver(prob)
    try:
        s.run(T=prob.params.T, max_steps=0)
        q, at, me = s.q(), s.arrival_times(), s.maximum_elevation()
    finally:
        s.close()
    np.testing.assert_array_equal(q, q_ref)
    np.testing.assert_array_equal(at, z["ArrivalTimings"])
    np.testing.assert_array_equal(me, z["MaximumElevation"])


@pytest.mark.parametrize("flags", [(1, 1), (1, 0), (0, 1)])
def test_engine_analysis_matches_oracle_on_curved_lake(flags):
    pr = problems.curved_lake(N=4, nel=16, steps=37)
    pr.params.ArrivalTimings, pr.params.maximumElevation = flags
    pr.params.h_0 = 1.0  # still-water level of the lake
    ref = OracleProblem(pr).run(max_steps=37)
    s = Solver(pr)
    try:
        t, steps = s.run(max_steps=37)
        q = s.q()
        at = s.arrival_times() if flags[0] else None
        me = s.maximum_elevation() if flags[1] else None
        for on, get in zip(flags, (s.arrival_times, s.maximum_elevation)):
            if not on:
                with pytest.raises(EsdgError) as ei:
                    get()
                assert ei.value.code == E_ARG
    finally:
        s.close()
    assert steps == ref["steps"] == 37 and t == ref["t"]
    np.testing.assert_array_equal(q, ref["q"])
    if flags[0]:
        np.testing.assert_array_equal(at, ref["ArrivalTimings"])
        assert 0 < (at == 1000.0).sum() < at.size
    if flags[1]:
        np.testing.assert_array_equal(me, ref["MaximumElevation"])
        assert me.max() > 0.0
