"""Serving loop on the GPU: a request's result is the same alone and in the
mix (bit for bit: every instance of the arena has its own time step and no
kernel mixes instances' numbers), requests are admitted while others are on
the GPU, and the learned indicator path stays within the stated deviation
of the plain one-at-a-time path."""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import serving
from esdgsem_mpiocca_b200.deviceclass import Solver
from esdgsem_mpiocca_b200.indicator import IndicatorNet

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-3


def _small_stream(n=6, seed=5):
    return serving.make_requests(n, rate=1e6, seed=seed, sizes=(32, 48, 64), horizons=(30, 90))


def test_alone_and_in_mix_are_identical_and_batching_is_continuous():
    reqs = _small_stream()
    # room for about two requests per degree: the rest wait and are
    # admitted as others finish
    srv = serving.Server(elements=5000, max_instances=8, chunk=2)
    stats = serving.serve(reqs, srv, realtime=False)
    srv.close()
    assert stats["requests"] == len(reqs) and stats["errors"] == 0
    adm = sorted(r.admitted for r in reqs)
    fin = sorted(r.finished for r in reqs)
    assert adm[-1] > fin[0]                       # someone was admitted after another finished
    assert any(r.admitted < s.finished and r.admitted > s.admitted for r in reqs for s in reqs)
    for r in reqs:
        one = serving.make_requests(len(reqs), rate=1e6, seed=5, sizes=(32, 48, 64), horizons=(30, 90))[r.rid]
        alone = serving.Server(elements=64 * 64, degrees=(r.N,), max_instances=1, chunk=3)
        serving.serve([one], alone, realtime=False)
        alone.close()
        np.testing.assert_array_equal(one.q, r.q)
        # the single-mesh engine with the same indicator gives the same numbers
        s = Solver(r.prob, indicator=2, net=IndicatorNet.default(r.N))
        s.run(T=1e9, max_steps=r.steps)
        np.testing.assert_array_equal(s.q(), r.q)
        s.close()


def test_served_results_stay_close_to_plain_solves():
    reqs = _small_stream(4, seed=9)
    srv = serving.Server(elements=4 * 64 * 64, max_instances=8)
    serving.serve(reqs, srv, realtime=False)
    srv.close()
    for r in reqs:
        s = Solver(r.prob)
        s.run(T=1e9, max_steps=r.steps)
        q0 = s.q().reshape(r.prob.K, 3, -1)
        s.close()
        q = r.q.reshape(r.prob.K, 3, -1)
        for v in range(3):
            assert np.linalg.norm(q[:, v] - q0[:, v]) <= TOL_L2 * np.linalg.norm(q0[:, v])


def test_realtime_stream_reports_latency():
    reqs = serving.make_requests(5, rate=50.0, seed=11, sizes=(32,), horizons=(20, 40))
    srv = serving.Server(elements=8 * 32 * 32, max_instances=8)
    st = serving.serve(reqs, srv, realtime=True)
    srv.close()
    assert st["requests"] == 5 and st["p99_s"] >= st["p50_s"] > 0
    assert all(r.admitted >= r.arrival for r in reqs)
