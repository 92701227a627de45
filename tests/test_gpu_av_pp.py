"""Artificial viscosity (shock sensor + BR1 gradient + viscous terms), the
positivity limiter and failure detection: CUDA engine vs CPU oracle (GPU).

Tolerances as in test_gpu_parity.py; the element viscosity is compared with
rtol 1e-13 (log10 and sin of CUDA and glibc may differ in the last ulp).
"""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.deviceclass import E_NONFINITE, EsdgError, Solver
from oracle.oracle import OracleProblem
from tests.test_gpu_parity import assert_rhs_close, rel_l2_per_var

pytestmark = pytest.mark.gpu


def small_dam(**kw):
    return problems.dam_break(N=kw.pop("N", 4), nel=kw.pop("nel", 12), seed=kw.pop("seed", 2), **kw)


def test_shock_sensor_ramps():
    pr = small_dam(steps=0)
    _, visc = OracleProblem(pr).rhs(pr.q0)
    p = pr.params
    # every branch of the sensor (zero, sine ramp, saturated) is hit
    assert (visc == 0).any()
    assert ((visc > 0) & (visc < p.epsilon_0)).any()


@pytest.mark.parametrize("N,rot", [(4, 0), (3, 5)])
def test_rhs_with_viscosity(N, rot):
    pr = small_dam(N=N, rotate_seed=rot, steps=0)
    s = Solver(pr)
    try:
        Qg, vg = s.rhs()
    finally:
        s.close()
    Qo, vo = OracleProblem(pr).rhs(pr.q0)
    np.testing.assert_allclose(vg, vo, rtol=1e-13, atol=1e-300)
    assert_rhs_close(Qg, Qo, pr)


def test_timeloop_with_viscosity_30_steps():
    pr = small_dam(steps=30)
    s = Solver(pr)
    try:
        t, steps = s.run()
        qg = s.q()
        vg = s.dc.copy_visc_to_host(pr.K)
    finally:
        s.close()
    ref = OracleProblem(pr).run()
    assert steps == ref["steps"] == 30
    assert abs(t - ref["t"]) <= 1e-12 * ref["t"]
    assert max(rel_l2_per_var(qg, ref["q"], pr.K, pr.ngl ** 2)) <= 1e-12
    np.testing.assert_allclose(vg, ref["visc"], rtol=1e-10, atol=1e-14)


def test_positivity_limiter_matches_oracle():
    pr = problems.periodic_bump(NumFlux=0, steps=3)
    pr.params.PositivityPreserving = 1
    pr.params.PosPresTOL = 1e-3
    q = pr.q0.reshape(pr.K, 3, -1).copy()
    # shallow elements with a diverging flow: the first stages drain them
    # below zero, so the limiter and the dry-momentum cut both act
    xi = np.tile(np.linspace(-1.0, 1.0, pr.ngl), pr.ngl)
    for e in (3, 77, 150):
        q[e, 0] = 0.01
        q[e, 1] = 0.01 * 5.0 * xi
    pr.q0 = q.reshape(-1)
    s = Solver(pr)
    try:
        s.run()
        qg = s.q()
    finally:
        s.close()
    ref = OracleProblem(pr).run()
    assert max(rel_l2_per_var(qg, ref["q"], pr.K, pr.ngl ** 2)) <= 1e-12
    assert (qg.reshape(pr.K, 3, -1)[:, 0] >= 0).all()


def test_nonfinite_state_reports_status_and_context_survives():
    pr = problems.periodic_bump(NumFlux=0, steps=5)
    q = pr.q0.copy()
    q[17] = np.nan
    s = Solver(pr, q0=q)
    try:
        with pytest.raises(EsdgError) as ei:
            s.run()
        assert ei.value.code == E_NONFINITE
    finally:
        s.close()
    # the CUDA context is still usable afterwards
    s2 = Solver(pr)
    try:
        t, steps = s2.run()
        assert steps == 5 and np.isfinite(s2.q()).all()
    finally:
        s2.close()
