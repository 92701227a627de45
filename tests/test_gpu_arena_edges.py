"""Edge cases of the batched ensemble with the indicator modes: capacity
and slot exhaustion, bad ids and unsupported learned degrees fail loudly;
an empty arena advances without work; an arena with the active set and
refills mid-flight gives each member exactly its alone result; the live
extent shrinks as the top member leaves without disturbing the others."""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.deviceclass import EsdgError, Solver
from esdgsem_mpiocca_b200.ensemble import Ensemble
from esdgsem_mpiocca_b200.indicator import IndicatorNet

pytestmark = pytest.mark.gpu


def _arena(probs, slots=None, slack=1.0):
    return Ensemble.for_problems(probs, max_instances=slots or len(probs), slack=slack)


def test_capacity_slots_and_bad_ids_fail_loudly():
    a = problems.dam_break(N=3, nel=16, seed=1)
    b = problems.dam_break(N=3, nel=24, seed=2)
    en = _arena([a], slots=2)
    en.add(a, T=1e9, max_steps=3)
    with pytest.raises(EsdgError):
        en.add(b, T=1e9, max_steps=3)      # no element range left
    with pytest.raises(EsdgError):
        en.remove(1)                       # never added
    en.close()
    en = _arena([a, a], slots=1)
    en.add(a, T=1e9, max_steps=3)
    with pytest.raises(EsdgError):
        en.add(a, T=1e9, max_steps=3)      # no slot left
    en.close()


def test_learned_indicator_rejects_unsupported_degree():
    p = problems.dam_break(N=2, nel=8, seed=3)
    en = _arena([p])
    with pytest.raises(EsdgError):
        en.set_indicator(2, IndicatorNet.default(3))
    en.close()


def test_empty_arena_advances_without_work():
    p = problems.dam_break(N=3, nel=8, seed=4)
    en = _arena([p])
    en.set_indicator(1)
    en.advance(3)
    en.add(p, T=1e9, max_steps=4)
    en.advance(2)
    assert en.status(0)["steps"] == 2
    en.close()


def test_active_set_arena_with_refills_matches_alone_runs():
    probs = [problems.dam_break(N=3, nel=16, seed=5), problems.bore(N=3, nel=16, seed=6),
             problems.dam_break(N=3, nel=12, seed=7), problems.bore(N=3, nel=12, seed=8)]
    steps = [12, 30, 20, 16]
    alone = []
    for p, n in zip(probs, steps):
        s = Solver(p)
        s.run(T=1e9, max_steps=n)
        alone.append(s.q())
        s.close()
    en = Ensemble.for_problems(probs[:3], max_instances=3, slack=1.0)
    en.set_indicator(1)
    ids = {k: en.add(probs[k], T=1e9, max_steps=steps[k]) for k in range(3)}
    got = {}
    pending = [3]
    while len(got) < 4:
        en.advance(2)
        for k, i in list(ids.items()):
            if en.status(i)["done"]:
                got[k] = en.q(i)
                en.remove(i)
                del ids[k]
        if pending:
            k = pending[0]
            K, F, slots = en.free_capacity()
            if slots and probs[k].K <= K and probs[k].F <= F:
                ids[k] = en.add(probs[k], T=1e9, max_steps=steps[k])
                pending.pop(0)
    en.close()
    for k in range(4):
        np.testing.assert_array_equal(got[k], alone[k])
