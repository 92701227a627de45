"""Host logic of the serving loop (esdgsem_mpiocca_b200/serving.py) with a
fake arena: Poisson request stream, FIFO admission by free capacity (a
request that does not fit holds back the later ones of its degree),
retirement frees capacity, latency statistics."""
import numpy as np

from esdgsem_mpiocca_b200 import serving


def test_request_stream_is_seeded_and_poisson():
    a = serving.make_requests(400, rate=100.0, seed=3, build=False)
    b = serving.make_requests(400, rate=100.0, seed=3, build=False)
    assert [(r.arrival, r.N, r.nel, r.steps, r.seed) for r in a] == [(r.arrival, r.N, r.nel, r.steps, r.seed)
                                                                     for r in b]
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert abs(gaps.mean() - 0.01) < 0.0015
    assert {r.N for r in a} == {3, 4}
    assert set(r.nel for r in a) <= set(serving.SIZES)
    assert all(200 <= r.steps <= 2000 for r in a)


class _FakeProb:
    def __init__(self, K):
        self.K, self.F = K, 2 * K


class FakeServer:
    """Capacity in elements per degree; a request needs `steps` chunks."""

    def __init__(self, cap):
        self.cap = dict(cap)
        self.live = {N: {} for N in cap}
        self.log = []

    def try_admit(self, r, now):
        if r.prob.K > self.cap[r.N]:
            return False
        self.cap[r.N] -= r.prob.K
        self.live[r.N][r.rid] = [r, r.steps]
        r.admitted = now
        self.log.append(("admit", r.rid))
        return True

    def busy(self):
        return any(self.live[N] for N in self.live)

    def step(self, now_fn):
        done = []
        for N in self.live:
            for rid in list(self.live[N]):
                ent = self.live[N][rid]
                ent[1] -= 1
                if ent[1] == 0:
                    r = ent[0]
                    del self.live[N][rid]
                    self.cap[N] += r.prob.K
                    r.finished = now_fn()
                    self.log.append(("done", rid))
                    done.append(r)
        return done


def _reqs(spec):
    out = []
    for k, (N, K, steps) in enumerate(spec):
        r = serving.Request(k, 0.0, N, int(K ** 0.5), steps, k)
        r.prob = _FakeProb(K)
        out.append(r)
    return out


def test_fifo_admission_and_continuous_batching():
    reqs = _reqs([(3, 60, 3), (3, 50, 1), (3, 30, 1), (4, 90, 2), (4, 20, 1)])
    srv = FakeServer({3: 100, 4: 100})
    stats = serving.serve(reqs, srv, realtime=False)
    assert stats["requests"] == 5
    order = srv.log
    # degree 3: request 1 (50) does not fit next to 0 (60): it and the later
    # request 2 wait (FIFO) although 2 alone would fit
    assert order.index(("admit", 1)) > order.index(("done", 0))
    assert order.index(("admit", 2)) > order.index(("admit", 1))
    # degree 4 runs concurrently: request 4 is admitted when 3 is done
    assert ("admit", 3) in order[:3]
    assert order.index(("admit", 4)) > order.index(("done", 3))
    # request 0 keeps running while 3 retires and 4 is admitted: batching
    # continues across retirements
    assert order.index(("admit", 4)) < order.index(("done", 0))
    assert all(r.latency >= 0 for r in reqs)


def test_shortest_job_first_order():
    # all arrive at t=0; capacity for one request at a time per degree
    reqs = _reqs([(3, 100, 4), (3, 100, 1), (3, 100, 2)])
    srv = FakeServer({3: 100})
    serving.serve(reqs, srv, realtime=False, policy="sjf")
    admits = [rid for kind, rid in srv.log if kind == "admit"]
    assert admits == [1, 2, 0]      # by work (steps at equal size)
    fifo = FakeServer({3: 100})
    serving.serve(serving.fresh(reqs), fifo, realtime=False, policy="fifo")
    assert [rid for kind, rid in fifo.log if kind == "admit"] == [0, 1, 2]


class _FakeArena:
    def __init__(self, K):
        self.K, self.n = K, 0

    def free_capacity(self):
        return self.K, 2 * self.K, 8

    def add(self, prob, T=None, max_steps=None):
        self.K -= prob.K
        self.n += 1
        return self.n


def test_live_node_cap():
    srv = serving.Server.__new__(serving.Server)
    srv.arenas = {3: _FakeArena(10 ** 6)}
    srv.live = {3: {}}
    srv.max_live_nodes = 2 * 64 * 64 * 16
    a, b, c = _reqs([(3, 64 * 64, 5), (3, 64 * 64, 5), (3, 64 * 64, 5)])
    assert srv.try_admit(a, 0.0) and srv.try_admit(b, 0.0)
    assert not srv.try_admit(c, 0.0)        # would exceed the nodes in flight
    srv.live[3].clear()
    big = _reqs([(3, 256 * 256, 5)])[0]
    assert srv.try_admit(big, 0.0)          # an idle server admits any request that fits
