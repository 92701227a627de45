"""The trained indicator networks (esdgsem_mpiocca_b200/weights) in the
solver, measured against the modal sensor on seeds the training never saw:

* flag agreement: on snapshots of a plain-sensor run, the viscosity the
  learned indicator assigns (network where confident, modal sensor
  elsewhere) against the modal sensor's, element by element;
* solution deviation: relative L2 difference per conserved variable between
  a learned-indicator run and the plain-sensor run from the same state
  (bound 1e-3);
* what the network gains: on the elements that are not trivially smooth
  (sensor value within two decades of the ramp), the trained network's
  prediction error and the share of them it settles correctly at its
  margin, against an untrained network and against the rule without a
  network (sigma_hat = s_eta, the log energy fraction alone).
"""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.deviceclass import Solver
from esdgsem_mpiocca_b200.indicator import IndicatorNet

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-3


def _rel_l2(a, b, K, n2):
    a = a.reshape(K, 3, n2)
    b = b.reshape(K, 3, n2)
    return [float(np.linalg.norm(a[:, v] - b[:, v]) / np.linalg.norm(b[:, v])) for v in range(3)]


def _agreement(prob, net, snapshots, every):
    """Flag agreement and decision shares over snapshots of a plain run."""
    ref = Solver(prob)
    ref.run(max_steps=every)
    agree, same, total = 0, 0, 0
    net_decided = 0
    for k in range(snapshots):
        q = ref.q()
        s0 = Solver(prob, q0=q)
        _, v0 = s0.rhs()
        s0.close()
        s2 = Solver(prob, q0=q, indicator=2, net=net)
        _, v2 = s2.rhs()
        st = s2.dc.indicator_stats()
        s2.close()
        agree += int(((v0 > 0) == (v2 > 0)).sum())
        same += int((v0 == v2).sum())
        total += prob.K
        net_decided += st["net_zero"] + st["net_full"]
        if k + 1 < snapshots:
            ref.dc.advance(every, 1e9)
    ref.close()
    return agree / total, same / total, net_decided / total


@pytest.mark.parametrize("N,make", [
    (4, lambda: problems.dam_break(N=4, nel=64, seed=1001)),
    (4, lambda: problems.bore(N=4, nel=64, seed=1002)),
    (3, lambda: problems.tsunami_member(1003, sizes=(64,))),
])
def test_learned_indicator_against_modal_sensor(N, make):
    prob = make()
    net = IndicatorNet.default(N)
    agree, same, decided = _agreement(prob, net, snapshots=6, every=40)
    assert agree >= 0.999, agree
    assert same >= 0.99, same
    assert decided >= 0.4, decided           # the network settles most elements


@pytest.mark.parametrize("N,make,steps", [
    (4, lambda: problems.dam_break(N=4, nel=64, seed=1004), 400),
    (3, lambda: problems.tsunami_member(1005, sizes=(64,)), 300),
])
def test_learned_run_deviation_is_within_tolerance(N, make, steps):
    prob = make()
    n2 = (N + 1) ** 2
    s0 = Solver(prob)
    s0.run(max_steps=steps)
    q0 = s0.q()
    s0.close()
    s2 = Solver(prob, indicator=2, net=IndicatorNet.default(N))
    s2.run(max_steps=steps)
    q2 = s2.q()
    st = s2.dc.indicator_stats()
    s2.close()
    dev = _rel_l2(q2, q0, prob.K, n2)
    assert max(dev) <= TOL_L2, dev
    assert st["net_zero"] + st["net_full"] > 0


@pytest.mark.parametrize("N,make,steps", [
    (3, lambda: problems.tsunami_member(1005, sizes=(64,)), 300),
])
def test_learned_once_per_step_deviation_is_within_tolerance(N, make, steps):
    """The learned indicator evaluated once per step (its viscosity and
    active set kept for the step's stages) on a tsunami member: the run
    stays within the same bound of the plain-sensor run, with fewer
    indicator launches.  (On the N = 4 dam break, whose shocks change the
    viscosity within a step, this schedule deviates by about 1e-2, outside
    the bound: it is an option, not the default.)"""
    prob = make()
    n2 = (N + 1) ** 2
    s0 = Solver(prob)
    s0.run(max_steps=steps)
    q0 = s0.q()
    s0.close()
    launches = {}
    q = {}
    for every in (True, False):
        s2 = Solver(prob, indicator=2, net=IndicatorNet.default(N))
        s2.dc.set_indicator_every_stage(every)
        l0 = s2.dc.kernel_launches()
        s2.run(max_steps=steps)
        launches[every] = s2.dc.kernel_launches() - l0
        q[every] = s2.q()
        s2.close()
    dev = _rel_l2(q[False], q0, prob.K, n2)
    assert max(dev) <= TOL_L2, dev
    assert launches[False] < launches[True]
    assert np.isfinite(q[False]).all()


def _snapshots(prob, every, count):
    """Feature rows, targets and s_eta of the elements of a plain run."""
    import torch
    from esdgsem_mpiocca_b200.indicator import DeviceMLP
    mlp = DeviceMLP(IndicatorNet.fresh(prob.params.N + 1), 0)
    sol = Solver(prob)
    sol.run(max_steps=every)
    Xs, ts, ss = [], [], []
    for k in range(count):
        qp, bp, vp = sol.dc.state_pointers()
        X, t, s = mlp.features(qp, bp, vp, prob.K)
        Xs.append(X), ts.append(t), ss.append(s)
        torch.cuda.synchronize()
        if k + 1 < count:
            sol.dc.advance(every, 1e9)
    sol.close()
    X, t, s = torch.cat(Xs), torch.cat(ts), torch.cat(ss)
    ok = torch.isfinite(t)
    return X[ok], t[ok], s[ok]


@pytest.mark.parametrize("N,make", [
    (4, lambda: problems.dam_break(N=4, nel=96, seed=3001)),
    (4, lambda: problems.bore(N=4, nel=96, seed=3002)),
    (3, lambda: problems.tsunami_member(3003, sizes=(96,))),
])
def test_trained_network_gain(N, make):
    import torch
    from esdgsem_mpiocca_b200.indicator import DeviceMLP
    prob = make()
    p = prob.params
    X, t, s = _snapshots(prob, 40, 6)
    sig = (t + s).double()
    crit = (sig > p.sigma_min - 2.0) & (sig < p.sigma_max + 2.0)
    assert int(crit.sum()) > 500
    net = IndicatorNet.default(N)
    m = net.margin
    out = {}
    for name, n in (("trained", net), ("untrained", IndicatorNet.fresh(N + 1, seed=0)), ("no_net", None)):
        y = DeviceMLP(n, 0).forward(X).double() if n is not None else torch.zeros_like(sig)
        sh = y + s.double()
        zero = sh < p.sigma_min - m
        full = sh > p.sigma_max + m
        right = (zero & (sig <= p.sigma_min)) | (full & (sig >= p.sigma_max))
        wrong = (zero | full) & ~right
        out[name] = dict(rmse=float(torch.sqrt(((sh - sig)[crit] ** 2).mean())),
                         settled=float(right[crit].double().mean()), wrong=float(wrong[crit].double().mean()))
    tr = out["trained"]
    assert tr["wrong"] <= 1e-3, out
    for other in ("untrained", "no_net"):
        assert tr["rmse"] < 0.25 * out[other]["rmse"], out
        assert tr["settled"] > out[other]["settled"] or out[other]["wrong"] > 10 * max(tr["wrong"], 1e-4), out
