"""Active set of the artificial-viscosity path (indicator modes 1 and 2)
against the reference-equivalent path (mode 0: the modal sensor and the
viscous terms on every element).

The viscous terms of an element are exactly zero unless it or a face
neighbour has viscosity > 0, so running the BR1 gradient and the viscous
kernels only on the flagged elements must give bit-identical solutions:
for the low-storage and SSP integrators, with the positivity limiter, for a
single right-hand side, and in the batched ensemble.  The learned mode with
an infinite margin hands every element to the modal sensor and must also
be bit-identical."""
import dataclasses

import numpy as np
import pytest

from esdgsem_mpiocca_b200 import host, problems
from esdgsem_mpiocca_b200.deviceclass import Solver
from esdgsem_mpiocca_b200.ensemble import Ensemble
from esdgsem_mpiocca_b200.indicator import IndicatorNet

pytestmark = pytest.mark.gpu


def _variant(prob, **kw):
    p = dataclasses.replace(prob.params, **kw)
    return host.make_problem(p, prob.mesh, prob.b, prob.q0, prob.meta)


def _run(prob, steps, indicator, net=None):
    s = Solver(prob, indicator=indicator, net=net)
    s.run(max_steps=steps)
    q = s.q()
    stats = s.dc.indicator_stats() if indicator else None
    s.close()
    return q, stats


CASES = {
    "dam_break_lsrk": lambda: problems.dam_break(N=4, nel=24, seed=1),
    "dam_break_ssp_pp": lambda: _variant(problems.dam_break(N=3, nel=20, seed=2), rkSSP=1, rkOrder=3,
                                         PositivityPreserving=1),
    "bore_N3": lambda: problems.bore(N=3, nel=24, seed=3),
    "tsunami": lambda: problems.tsunami_member(7, sizes=(64,)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_active_set_is_bit_identical(name):
    prob = CASES[name]()
    q0, _ = _run(prob, 40, 0)
    q1, st = _run(prob, 40, 1)
    assert np.isfinite(q0).all()
    assert not np.array_equal(q0, prob.q0)
    np.testing.assert_array_equal(q1, q0)
    # the set is sparse: most elements skip the viscous kernels
    stages = 40 * len(prob.rkA)
    assert st["modal"] == stages * prob.K
    assert 0 < st["viscous"] < 0.9 * stages * prob.K


def test_learned_mode_with_infinite_margin_is_bit_identical():
    prob = problems.dam_break(N=4, nel=24, seed=4)
    net = IndicatorNet.fresh(5, seed=0)
    net.margin = 1e30
    q0, _ = _run(prob, 30, 0)
    q2, st = _run(prob, 30, 2, net)
    np.testing.assert_array_equal(q2, q0)
    assert st["net_zero"] == 0 and st["net_full"] == 0 and st["modal"] == 30 * 5 * prob.K


def test_rhs_is_bit_identical():
    prob = problems.dam_break(N=4, nel=16, seed=5)
    s0 = Solver(prob)
    s0.run(max_steps=25)
    q = s0.q()
    Qt0, v0 = s0.rhs()
    s0.close()
    s1 = Solver(prob, q0=q, indicator=1)
    Qt1, v1 = s1.rhs()
    s1.close()
    np.testing.assert_array_equal(v1, v0)
    np.testing.assert_array_equal(Qt1, Qt0)


def test_ensemble_active_set_is_bit_identical():
    probs = [problems.dam_break(N=3, nel=16, seed=6), problems.bore(N=3, nel=20, seed=7),
             problems.dam_break(N=3, nel=12, seed=8)]
    out = []
    for mode in (0, 1):
        en = Ensemble.for_problems(probs)
        if mode:
            en.set_indicator(1)
        ids = [en.add(p, T=1e9, max_steps=30 + 5 * k) for k, p in enumerate(probs)]
        en.run_until_done(ids)
        out.append([en.q(i) for i in ids])
        en.close()
    for a, b in zip(*out):
        np.testing.assert_array_equal(b, a)


def test_indicator_needs_artificial_viscosity():
    from esdgsem_mpiocca_b200.deviceclass import EsdgError
    prob = problems.periodic_bump(steps=2)
    with pytest.raises(EsdgError):
        Solver(prob, indicator=1)


@pytest.mark.parametrize("make", [
    lambda: problems.tsunami_member(11, sizes=(64,)),
    lambda: problems.dam_break(N=3, nel=32, seed=5),
    lambda: problems.dam_break(N=4, nel=24, seed=6),
    lambda: problems.tsunami_member(12, sizes=(32,), N=4),
    # element counts whose last tile of the fused pass ends inside a warp
    # (441 = 6 * 64 + 57 at N = 3, 529 = 16 * 32 + 17 at N = 4): idle
    # element slots next to live ones in the same network tile
    lambda: problems.dam_break(N=3, nel=21, seed=5),
    lambda: problems.dam_break(N=4, nel=23, seed=6),
])
def test_fused_learned_pass_equals_three_passes(make):
    """Mode 2 at N = 3 and 4 runs features, network and sensor fallback as
    one fused kernel; mode 3 runs the three separate passes.  Same
    decisions, same solution, bit for bit."""
    prob = make()
    net = IndicatorNet.default(prob.params.N)
    q2, st2 = _run(prob, 30, 2, net)
    q3, st3 = _run(prob, 30, 3, net)
    np.testing.assert_array_equal(q2, q3)
    assert st2 == st3
    assert st2["net_zero"] + st2["net_full"] > 0


def test_fused_learned_pass_in_the_arena():
    from esdgsem_mpiocca_b200.ensemble import Ensemble
    probs = [problems.tsunami_member(s, sizes=(32,)) for s in (21, 22, 23)]
    steps = [25, 15, 20]
    out = {}
    for mode in (2, 3):
        ens = Ensemble.for_problems(probs)
        try:
            ens.set_indicator(mode, IndicatorNet.default(3))
            ids = [ens.add(p, T=1e9, max_steps=s) for p, s in zip(probs, steps)]
            ens.run_until_done(ids)
            out[mode] = ([ens.q(i) for i in ids], ens.indicator_stats())
        finally:
            ens.close()
    for a, b in zip(out[2][0], out[3][0]):
        np.testing.assert_array_equal(a, b)
    assert out[2][1] == out[3][1]
