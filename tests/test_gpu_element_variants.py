"""Every element-kernel variant computes the same bits (GPU).

The engine compiles several variants of its element kernel (one thread per
node with different occupancy / pipeline depth; one thread per element line
evaluating each symmetric two-point flux once) and lets an autotuner pick
the fastest.  Each variant is fixed in turn here and must reproduce variant
0 bit for bit: in the LS-RK update, the SSP update with the positivity
limiter, the RHS-only mode, with artificial viscosity on the active set
(flagged elements leave through Qt), and in the batched arena (instances
that finish early leave tiles with inactive elements).
"""
import dataclasses

import numpy as np
import pytest

from esdgsem_mpiocca_b200 import host, problems
from esdgsem_mpiocca_b200.deviceclass import EsdgError, Solver, E_UNSUPPORTED
from esdgsem_mpiocca_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def _variant(prob, **kw):
    p = dataclasses.replace(prob.params, **kw)
    return host.make_problem(p, prob.mesh, prob.b, prob.q0, prob.meta)


def _usable(dc):
    """Variants available for this mesh (needs one tuned or fixed run)."""
    info = dc.element_variants()
    assert info is not None
    return [v for v, c in enumerate(info["ctas_per_sm"]) if c > 0]


def _run(prob, variant, steps, indicator=0):
    s = Solver(prob, indicator=indicator)
    try:
        s.dc.set_element_variant(variant)
        s.run(T=1e9, max_steps=steps)
        info = s.dc.element_variants()
        assert info["chosen"] == variant
        return s.q()
    finally:
        s.close()


def _variants_of(prob):
    s = Solver(prob)
    try:
        s.dc.set_element_variant(0)
        vs = _usable(s.dc)
    finally:
        s.close()
    return vs


CASES = {
    "lake_N4_lsrk": (lambda: problems.curved_lake(N=4, nel=34, seed=3, ripple=0.05, rotate_seed=2), 12, 0),
    "periodic_N3_nf2": (lambda: problems.periodic_bump(N=3, nel=18, NumFlux=2), 15, 0),
    "lake_N2_nf3": (lambda: problems.curved_lake(N=2, nel=22, seed=4, ripple=0.05, NumFlux=3), 10, 0),
    "lake_N5": (lambda: problems.curved_lake(N=5, nel=13, seed=5, ripple=0.05), 8, 0),
    "dam_ssp_pp_N3": (lambda: _variant(problems.dam_break(N=3, nel=20, seed=2), rkSSP=1, rkOrder=3,
                                       PositivityPreserving=1), 20, 0),
    "dam_av_full_N4": (lambda: problems.dam_break(N=4, nel=24, seed=1), 15, 0),
    "dam_av_active_set_N4": (lambda: problems.dam_break(N=4, nel=24, seed=1), 15, 1),
}


@pytest.mark.parametrize("name", list(CASES))
def test_variants_bitwise_equal(name):
    make, steps, indicator = CASES[name]
    prob = make()
    vs = _variants_of(prob)
    assert 0 in vs
    ref = _run(prob, 0, steps, indicator)
    assert np.isfinite(ref).all()
    for v in vs[1:]:
        np.testing.assert_array_equal(_run(prob, v, steps, indicator), ref, err_msg=f"variant {v}")


def test_row_variants_exist_for_N3_N4():
    for N in (3, 4):
        vs = _variants_of(problems.curved_lake(N=N, nel=16, seed=0))
        assert {3, 4} <= set(vs), (N, vs)


def test_rhs_only_mode_bitwise_equal():
    prob = problems.curved_lake(N=4, nel=20, seed=8, ripple=0.1, rotate_seed=1)
    out = {}
    for v in _variants_of(prob):
        s = Solver(prob)
        try:
            s.dc.set_element_variant(v)
            out[v] = s.rhs()
        finally:
            s.close()
    for v, Q in out.items():
        np.testing.assert_array_equal(Q, out[0], err_msg=f"variant {v}")


def test_unavailable_variant_is_rejected():
    prob = problems.curved_lake(N=1, nel=8, seed=0)   # no line-per-thread kernel for N = 1
    s = Solver(prob)
    try:
        with pytest.raises(EsdgError) as ei:
            s.dc.set_element_variant(3)
        assert ei.value.code == E_UNSUPPORTED
        with pytest.raises(EsdgError):
            s.dc.set_element_variant(99)
    finally:
        s.close()


def test_arena_variants_bitwise_equal():
    probs = [problems.periodic_bump(N=3, NumFlux=0, steps=0),
             problems.curved_lake(N=3, nel=10, seed=2, ripple=0.05, NumFlux=0, rotate_seed=4),
             problems.curved_lake(N=3, nel=7, seed=6, ripple=0.08, NumFlux=0)]
    steps = [30, 12, 21]
    results = {}
    for v in (0, 1, 2, 3, 4):
        ens = Ensemble.for_problems(probs)
        try:
            ens.set_element_variant(v)
            ids = [ens.add(p, T=1e9, max_steps=s) for p, s in zip(probs, steps)]
            ens.run_until_done(ids)
            assert ens.element_variants()["chosen"] == v
            results[v] = [ens.q(i) for i in ids]
        finally:
            ens.close()
    for v in results:
        for a, b in zip(results[v], results[0]):
            np.testing.assert_array_equal(a, b, err_msg=f"variant {v}")
