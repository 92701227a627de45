"""The engine at every degree it accepts, against the oracle (GPU).

N = 1, 2, 5, 6 and 7 on rotated curved meshes (every face-orientation
pairing), with the problems of tests/test_reference_live_cpu.py, where the
oracle ends in the reference program's state bit for bit; so engine ==
oracle here is engine == reference.  Per degree: one right-hand side
(max|dQt| <= 1e-13 of the largest term), the run to T = 0.01 the live pin
uses, and 100 LS-RK4 steps (relative L2 per variable <= 1e-12, the same
step count and time).  The kernel of okl/DG/VolumeKernelFluxDiffV99.okl:60-218
is generic in the number of nodes per direction; every degree is compiled
as its own instantiation.
"""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.deviceclass import Solver
from oracle.oracle import OracleProblem
from tests.test_gpu_parity import assert_rhs_close, rel_l2_per_var

pytestmark = pytest.mark.gpu

# the live pins' problems (tests/test_reference_live_cpu.py)
CASES = {
    1: lambda: problems.curved_lake(N=1, nel=12, seed=8, ripple=0.05, rotate_seed=6),
    2: lambda: problems.curved_lake(N=2, nel=10, seed=9, ripple=0.05, NumFlux=3, rotate_seed=2),
    5: lambda: problems.curved_lake(N=5, nel=8, seed=5, ripple=0.05, rotate_seed=3),
    6: lambda: problems.curved_lake(N=6, nel=6, seed=6, ripple=0.05, NumFlux=3, rotate_seed=9),
    7: lambda: problems.curved_lake(N=7, nel=5, seed=7, ripple=0.05, rotate_seed=4),
}


@pytest.mark.parametrize("N", sorted(CASES))
def test_rhs_at_degree(N):
    pr = CASES[N]()
    assert (pr.mesh.EdgeReversed == 0).any()
    s = Solver(pr)
    try:
        Qg = s.rhs()
    finally:
        s.close()
    assert_rhs_close(Qg, OracleProblem(pr).rhs(pr.q0), pr)


@pytest.mark.parametrize("N", sorted(CASES))
def test_run_to_live_pin_time(N):
    pr = CASES[N]()
    s = Solver(pr)
    try:
        t, steps = s.run(T=0.01, max_steps=0)
        qg = s.q()
    finally:
        s.close()
    ref = OracleProblem(pr).run(T=0.01, max_steps=0)
    assert steps == ref["steps"] >= 3
    errs = rel_l2_per_var(qg, ref["q"], pr.K, pr.ngl ** 2)
    assert max(errs) <= 1e-12, errs


@pytest.mark.parametrize("N", sorted(CASES))
def test_100_steps_at_degree(N):
    pr = CASES[N]()
    s = Solver(pr)
    try:
        t, steps = s.run(T=1e9, max_steps=100)
        qg = s.q()
    finally:
        s.close()
    ref = OracleProblem(pr).run(T=1e9, max_steps=100)
    assert steps == ref["steps"] == 100
    assert abs(t - ref["t"]) <= 1e-13 * ref["t"]
    assert np.isfinite(qg).all()
    errs = rel_l2_per_var(qg, ref["q"], pr.K, pr.ngl ** 2)
    assert max(errs) <= 1e-12, errs
