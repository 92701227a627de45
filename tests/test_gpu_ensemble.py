"""Batched ensemble (arena) on the GPU: every instance advanced inside the
batch equals, bit for bit, the same problem advanced alone by the
single-mesh engine -- also when a finished instance is removed and a new one
is admitted into its freed range while the others keep running.
"""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.deviceclass import Solver
from esdgsem_mpiocca_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def alone(pr, steps):
    s = Solver(pr)
    try:
        t, n = s.run(T=1e9, max_steps=steps)
        return s.q(), t, n
    finally:
        s.close()


def members():
    return [problems.periodic_bump(N=3, NumFlux=0, steps=0),
            problems.curved_lake(N=3, nel=10, seed=2, ripple=0.05, NumFlux=0, rotate_seed=4),
            problems.curved_lake(N=3, nel=7, seed=6, ripple=0.08, NumFlux=0)]


def test_batched_instances_equal_alone_runs():
    probs = members()
    steps = [30, 12, 21]
    ens = Ensemble.for_problems(probs)
    try:
        ids = [ens.add(p, T=1e9, max_steps=s) for p, s in zip(probs, steps)]
        ens.run_until_done(ids)
        for i, p, s in zip(ids, probs, steps):
            st = ens.status(i)
            assert st["done"] and st["steps"] == s and st["status"] == 0
            q_alone, t_alone, _ = alone(p, s)
            assert st["t"] == t_alone
            np.testing.assert_array_equal(ens.q(i), q_alone)
    finally:
        ens.close()


def test_continuous_batching_refill_mid_flight():
    a, b, c = members()
    ens = Ensemble(3, max_instances=2, K_capacity=a.K + b.K, F_capacity=a.F + b.F)
    try:
        ia = ens.add(a, T=1e9, max_steps=5)
        ib = ens.add(b, T=1e9, max_steps=40)
        ens.run_until_done([ia], chunk=1)
        q_a = ens.q(ia)
        ens.remove(ia)
        ic = ens.add(c, T=1e9, max_steps=9)      # takes the freed slot and range
        ens.run_until_done([ib, ic], chunk=4)
        np.testing.assert_array_equal(q_a, alone(a, 5)[0])
        np.testing.assert_array_equal(ens.q(ib), alone(b, 40)[0])
        np.testing.assert_array_equal(ens.q(ic), alone(c, 9)[0])
    finally:
        ens.close()


def test_tsunami_member_alone_matches_oracle():
    """An ensemble member at its own scales (2000 km square, 4000 m shelf,
    Okada uplift, artificial viscosity) run alone by the engine against the
    oracle (which equals the reference program on it bit for bit,
    tests/test_reference_live_cpu.py): relative L2 per variable <= 1e-12
    (the shock sensor's log10 and sin differ in the last ulp between CUDA
    and glibc)."""
    from oracle.oracle import OracleProblem
    pr = problems.tsunami_member(3, N=3, steps=0, sizes=(16,))
    s = Solver(pr)
    try:
        t, n = s.run(T=300.0, max_steps=0)
        q = s.q()
    finally:
        s.close()
    ref = OracleProblem(pr).run(T=300.0, max_steps=0)
    assert n == ref["steps"] >= 3 and t == pytest.approx(300.0, abs=1e-9)
    K, n2 = pr.K, pr.ngl ** 2
    a, b = q.reshape(K, 3, n2), ref["q"].reshape(K, 3, n2)
    for v in range(3):
        err = np.linalg.norm(a[:, v] - b[:, v]) / np.linalg.norm(b[:, v])
        assert err <= 1e-12, (v, err)
