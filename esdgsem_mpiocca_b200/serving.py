"""Continuous-batching solve server on the batched ensemble engine.

Requests (one shallow-water solve each: a mesh, an initial state, a step
horizon) arrive over time; the server keeps one arena per polynomial degree
resident on the GPU, admits a waiting request as soon as its element and
face ranges fit in the arena's free HBM capacity and an instance slot is
free, advances every admitted request together (one graph replay per step
for the whole arena, each request with its own time step), and retires each
request the moment its horizon is reached -- freeing its capacity for the
next one while the others keep running.  No counterpart in the reference.

Admission order: first-in first-out (a request that does not fit blocks the
later ones of its degree), or shortest job first (waiting requests ordered
by their work, K (N+1)^2 x 5 x steps DOF-stages, each admitted as soon as it
fits).  A cap on the nodes in flight (`max_live_nodes`) keeps the GPU
busy without spreading it over more requests than it needs: once one
request fills the GPU, every further concurrent request only slows all of
them down.

The one-at-a-time baseline serves the same stream first-in first-out with
one single-mesh solver per request (the plain path: modal sensor and viscous
terms on every element).

Request generator (the serving configuration): seeded tsunami scenarios of
the ensemble generator with K = nel^2, nel in {32, 64, 96, 128, 192, 256},
N in {3, 4}, horizons of 200-2000 steps, Poisson arrivals at a given rate.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np

from . import problems
from .deviceclass import Solver
from .ensemble import Ensemble
from .host import Problem
from .indicator import IndicatorNet

SIZES = (32, 64, 96, 128, 192, 256)
DEGREES = (3, 4)
HORIZONS = (200, 2000)


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float          # seconds after the stream starts
    N: int
    nel: int
    steps: int
    seed: int
    prob: Problem | None = None
    # filled by the server
    admitted: float = float("nan")
    finished: float = float("nan")
    q: np.ndarray | None = None
    status: int = 0

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    def dof_stages(self) -> float:
        return float(self.nel * self.nel * (self.N + 1) ** 2 * 5 * self.steps)

    @property
    def nodes(self) -> int:
        return self.nel * self.nel * (self.N + 1) ** 2


def make_requests(n: int, rate: float, seed: int = 0, sizes=SIZES, degrees=DEGREES, horizons=HORIZONS,
                  build: bool = True) -> list[Request]:
    """n requests with exponential inter-arrival times of mean 1/rate."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        nel = int(rng.choice(sizes))
        N = int(rng.choice(degrees))
        steps = int(rng.integers(horizons[0], horizons[1] + 1))
        sd = int(rng.integers(0, 2 ** 31 - 1))
        r = Request(k, t, N, nel, steps, sd)
        if build:
            r.prob = problems.tsunami_member(sd, N=N, steps=steps, sizes=(nel,))
        out.append(r)
    return out


def arena_bytes_per_unit(N: int, device_id: int = -1) -> tuple[float, float]:
    """Device bytes of the arena per element and per face (from two small
    arenas; includes the indicator's buffers)."""
    def size(Kc, Fc):
        en = Ensemble(N, 4, Kc, Fc, ArtificialViscosity=1, epsilon_0=1.0, sigma_max=-3.0, sigma_min=-7.0,
                      device_id=device_id)
        en.set_indicator(2, IndicatorNet.default(N))
        b = en.bytes()
        en.close()
        return b
    b0 = size(4096, 4096)
    bk = size(8192, 4096) - b0
    bf = size(4096, 8192) - b0
    return bk / 4096.0, bf / 4096.0


class Server:
    """One arena per polynomial degree, sized from an HBM budget (bytes)."""

    def __init__(self, hbm_bytes: float | None = None, degrees=DEGREES, max_instances: int = 256,
                 indicator: int = 2, device_id: int = -1, chunk: int = 4, params: Problem | None = None,
                 elements: int | None = None, max_live_nodes: int | None = None,
                 chunk_node_steps: float = 2e7, max_chunk: int = 64):
        """Arena capacity per degree from an HBM budget (split evenly across
        the degrees), or `elements` per arena directly.  max_live_nodes:
        admit a request only while the nodes of the live requests stay
        within this (a request is always admitted into an idle server).
        Steps per host poll: at least `chunk`, and with little work in
        flight up to `max_chunk`, so that a poll covers about
        `chunk_node_steps` node updates (the poll's host round trip is then
        small against the GPU time it covers)."""
        self.chunk = chunk
        self.chunk_node_steps = chunk_node_steps
        self.max_chunk = max_chunk
        self.max_live_nodes = max_live_nodes
        self.arenas: dict[int, Ensemble] = {}
        self.live: dict[int, dict[int, Request]] = {}
        p = (params or problems.tsunami_member(0, sizes=(8,))).params
        for N in degrees:
            if elements is None:
                be, bf = arena_bytes_per_unit(N, device_id)
                # faces ~ 2 per element on the generator's meshes
                Kc = int(hbm_bytes / len(degrees) / (be + 2.05 * bf))
            else:
                Kc = int(elements)
            Fc = int(2.05 * Kc) + 64
            en = Ensemble(N, max_instances, Kc, Fc, NumFlux=p.NumFlux, g_const=p.g_const, PosPresTOL=p.PosPresTOL,
                          ArtificialViscosity=1, epsilon_0=p.epsilon_0, sigma_max=p.sigma_max,
                          sigma_min=p.sigma_min, device_id=device_id)
            en.set_indicator(indicator, IndicatorNet.default(N) if indicator == 2 else None)
            self.arenas[N] = en
            self.live[N] = {}

    def capacity(self):
        return {N: en.free_capacity() for N, en in self.arenas.items()}

    def live_nodes(self) -> int:
        return sum(r.nodes for live in self.live.values() for r in live.values())

    def try_admit(self, r: Request, now: float) -> bool:
        if self.max_live_nodes is not None and self.busy() and self.live_nodes() + r.nodes > self.max_live_nodes:
            return False
        en = self.arenas[r.N]
        K, F = r.prob.K, r.prob.F
        ke, kf, slots = en.free_capacity()
        if slots == 0 or K > ke or F > kf:
            return False
        i = en.add(r.prob, T=1e9, max_steps=r.steps)
        self.live[r.N][i] = r
        r.admitted = now
        return True

    def busy(self) -> bool:
        return any(self.live[N] for N in self.live)

    def step(self, now_fn) -> list[Request]:
        """Advances every arena with live requests by `chunk` steps and
        retires the finished ones (results copied out, capacity freed)."""
        done = []
        running = [N for N in self.arenas if self.live[N]]
        live = max(self.live_nodes(), 1)
        chunk = max(self.chunk, min(self.max_chunk, int(self.chunk_node_steps / live)))
        for N in running:  # the arenas run concurrently, each on its own stream
            self.arenas[N].launch(chunk)
        for N in running:
            en = self.arenas[N]
            en.sync()
            for i in list(self.live[N]):
                s = en.status(i)
                if s["done"]:
                    r = self.live[N].pop(i)
                    r.q = en.q(i)
                    r.status = s["status"]
                    en.remove(i)
                    r.finished = now_fn()
                    done.append(r)
        return done

    def close(self):
        for en in self.arenas.values():
            en.close()
        self.arenas.clear()


def serve(requests: list[Request], server: Server, realtime: bool = True, policy: str = "fifo") -> dict:
    """Serves the stream: arrivals in (wall-clock) time, admission by free
    capacity in FIFO or shortest-job-first order, continuous batching.
    Returns latency statistics."""
    if policy not in ("fifo", "sjf"):
        raise ValueError("policy must be 'fifo' or 'sjf'")
    t0 = time.perf_counter()

    def now():
        return time.perf_counter() - t0

    pending = sorted(requests, key=lambda r: r.arrival)
    waiting: list[Request] = []
    finished: list[Request] = []
    k = 0
    while len(finished) < len(requests):
        t = now() if realtime else float("inf")
        while k < len(pending) and pending[k].arrival <= t:
            waiting.append(pending[k])
            k += 1
        rest = []
        if policy == "fifo":
            # a request that does not fit blocks the ones behind it of the
            # same degree, so large requests are not starved
            blocked = set()
            for r in waiting:
                if r.N in blocked or not server.try_admit(r, now()):
                    blocked.add(r.N)
                    rest.append(r)
        else:
            for r in sorted(waiting, key=lambda r: (r.dof_stages(), r.arrival)):
                if not server.try_admit(r, now()):
                    rest.append(r)
        waiting = rest
        if server.busy():
            finished.extend(server.step(now))
        elif k < len(pending) and realtime:
            time.sleep(max(0.0, min(pending[k].arrival - now(), 0.05)))
        elif waiting:
            raise RuntimeError(f"request {waiting[0].rid} does not fit an empty arena")
        else:
            break
    wall = now()
    return summarize(finished, wall)


def serve_one_at_a_time(requests: list[Request], indicator: int = 0, realtime: bool = True,
                        device_id: int = -1) -> dict:
    """The same stream served first-in first-out by single-mesh solvers, one
    request on the GPU at a time (indicator 0: the plain path)."""
    t0 = time.perf_counter()

    def now():
        return time.perf_counter() - t0

    finished = []
    for r in sorted(requests, key=lambda r: r.arrival):
        if realtime:
            w = r.arrival - now()
            if w > 0:
                time.sleep(w)
        r.admitted = now()
        net = IndicatorNet.default(r.N) if indicator == 2 else None
        s = Solver(r.prob, device_id=device_id, indicator=indicator, net=net)
        s.run(T=1e9, max_steps=r.steps)
        r.q = s.q()
        s.close()
        r.finished = now()
        finished.append(r)
    return summarize(finished, now())


def fresh(requests: list[Request]) -> list[Request]:
    """Copies of the requests (same inputs) without any served results."""
    return [Request(r.rid, r.arrival, r.N, r.nel, r.steps, r.seed, r.prob) for r in requests]


def summarize(finished: list[Request], wall: float) -> dict:
    lat = np.array([r.latency for r in finished])
    work = sum(r.dof_stages() for r in finished)
    return {"requests": len(finished), "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None, "mean_s": float(lat.mean()),
            "wall_s": wall, "throughput_dof_stages_per_s": work / wall, "requests_per_s": len(finished) / wall,
            "errors": sum(1 for r in finished if r.status != 0)}
