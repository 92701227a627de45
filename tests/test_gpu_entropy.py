"""Entropy behaviour of the engine's scheme: with the interface dissipation switched off (ES=0) the
semi-discrete scheme conserves the total entropy
    S = sum_e sum_ij J w_i w_j ( h (u^2 + v^2) / 2 + g h^2 / 2 + g h b )
to round-off, i.e. the entropy variables w = (g (h + b) - (u^2 + v^2) / 2,
u, v) contracted with the right-hand side L(q) under the LGL quadrature
vanish up to rounding of the terms; with ES=1 the rate is negative.  Over a
run the total entropy then changes only by the time-integration error
(ES=0), and decreases (ES=1)."""
import dataclasses

import numpy as np
import pytest

from esdgsem_mpiocca_b200 import host, problems
from esdgsem_mpiocca_b200.deviceclass import Solver

pytestmark = pytest.mark.gpu


def _variant(prob, **kw):
    p = dataclasses.replace(prob.params, **kw)
    return host.make_problem(p, prob.mesh, prob.b, prob.q0, prob.meta)


def _rate(prob, q=None):
    """(dS/dt, sum of |terms|) for the engine's RHS at state q."""
    s = Solver(prob, q0=q)
    Qt = s.rhs()
    s.close()
    n2 = prob.ngl ** 2
    K = prob.K
    qq = (prob.q0 if q is None else q).reshape(K, 3, n2)
    Qt = Qt.reshape(K, 3, n2)
    h, hu, hv = qq[:, 0], qq[:, 1], qq[:, 2]
    u, v = hu / h, hv / h
    g = prob.params.g_const
    b = prob.b.reshape(K, n2)
    w0 = g * (h + b) - 0.5 * (u * u + v * v)
    wq = np.outer(prob.basis.wGL, prob.basis.wGL).reshape(n2)   # node (xi, eta): eta-major, symmetric weights
    Jw = wq[None, :] / prob.mesh.Jinv.reshape(K, n2)
    terms = Jw * (w0 * Qt[:, 0] + u * Qt[:, 1] + v * Qt[:, 2])
    return float(terms.sum()), float(np.abs(Jw * (np.abs(w0 * Qt[:, 0]) + np.abs(u * Qt[:, 1]) +
                                                   np.abs(v * Qt[:, 2]))).sum())


def _perturbed(prob, seed=0, amp=0.05, jumps=True):
    """A smooth flow, plus (jumps=True) element-wise offsets so that the
    traces jump across every interface (where the dissipation acts)."""
    rng = np.random.default_rng(seed)
    n2 = prob.ngl ** 2
    q = prob.q0.reshape(prob.K, 3, n2).copy()
    x, y = prob.mesh.x.reshape(prob.K, n2), prob.mesh.y.reshape(prob.K, n2)
    kx, ky = rng.integers(1, 4, size=2)
    q[:, 1] += amp * np.sin(np.pi * kx * x) * np.cos(np.pi * ky * y)
    q[:, 2] += amp * np.cos(np.pi * kx * x + 0.3)
    q[:, 0] += 0.3 * amp * np.sin(np.pi * (x + y))
    if jumps:
        q += 0.1 * amp * rng.normal(size=(prob.K, 3, 1))
    return q.reshape(-1)


@pytest.mark.parametrize("numflux", [0, 2, 3])
def test_entropy_rate_vanishes_without_dissipation(numflux):
    base = problems.periodic_bump(NumFlux=numflux)
    q = _perturbed(base, seed=numflux)
    ec = _variant(base, ES=0)
    rate, scale = _rate(ec, q)
    assert abs(rate) <= 1e-13 * scale, (rate, scale)
    es = _variant(base, ES=1)
    rate_es, scale_es = _rate(es, q)
    assert rate_es < -1e-9 * scale_es, (rate_es, scale_es)


def test_entropy_rate_vanishes_on_curved_walls():
    base = problems.curved_lake(N=4, nel=8, seed=2, ripple=0.05, rotate_seed=5)
    q = _perturbed(base, seed=7, amp=0.02)
    rate, scale = _rate(_variant(base, ES=0), q)
    assert abs(rate) <= 1e-13 * scale, (rate, scale)


def _entropy_change(pr, q, T):
    s0 = host.diagnostics(pr.mesh, pr.basis, q, b=pr.b, g=pr.params.g_const)["entropy"]
    s = Solver(pr, q0=q)
    s.run(T=T, max_steps=0)
    s1 = host.diagnostics(pr.mesh, pr.basis, s.q(), b=pr.b, g=pr.params.g_const)["entropy"]
    s.close()
    return (s1 - s0) / abs(s0)


def test_total_entropy_over_a_run():
    """Without dissipation the entropy of a smooth run changes only by the
    fourth-order time-integration error (halving the step divides it by
    about 16); with dissipation and jumps it decreases."""
    base = problems.periodic_bump(NumFlux=0)
    q = _perturbed(base, seed=3, jumps=False)
    T = 0.2
    d = {cfl: _entropy_change(_variant(base, ES=0, CFL=cfl), q, T) for cfl in (0.4, 0.2)}
    assert abs(d[0.4]) < 1e-8, d
    assert abs(d[0.2]) < abs(d[0.4]) / 8, d
    qj = _perturbed(base, seed=3)
    assert _entropy_change(_variant(base, ES=1), qj, T) < -1e-7
