"""The multi-GPU plumbing of bench.py on two CPU ranks (gloo): the timed
region's max over ranks and the whole-job sums used for `value`, the
replicas' job rate and the ensemble line's aggregation (batched rate over the
slowest rank, one-at-a-time rates summed, worst deviation) as bench.py calls
them, and the disjoint per-rank sharding of ensemble members (no data-path
exchange)."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import bench
    dist = bench.init_dist(ws, backend="gloo")
    try:
        ms_max = bench.max_over_ranks(10.0 + rank, dist, device="cpu")
        units = bench.sum_over_ranks(100.0 * (rank + 1), dist, device="cpu")
        seeds = bench.member_seeds(rank, 4)
        # replicas of the plain workload: 1000 (rank 0) and 3000 (rank 1)
        # DOF-stages in 2 and 4 ms -> 4000 over the slowest 4 ms
        rate = bench.job_rate(1000.0 * (2 * rank + 1), 2.0 * (rank + 1), dist, device="cpu")
        # ensemble shards: batched dofs 10/20 over 5 steps in 1/2 ms; each
        # rank's one-at-a-time sample 4/6 dofs in 3 ms; deviations 1e-9/2e-8
        ens = bench.ensemble_summary(10.0 * (rank + 1), 1.0 + rank, 5, 4.0 + 2 * rank, 3.0, (1e-9, 2e-8)[rank],
                                     dist, device="cpu")
        dist.barrier()
        out.put((rank, ms_max, units, seeds, bench.dist_env(), rate, ens))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_the_bench():
    ws = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, out)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms_max, units, seeds, env, rate, ens in res:
        assert ms_max == 11.0            # the slowest rank's time, seen by every rank
        assert units == 300.0            # whole-job work
        assert env == (ws, rank, rank)
        assert abs(rate - 4000.0 / 4e-3) < 1e-6 * rate
        b, alone, dev = ens
        import bench
        S = bench.STAGES
        assert abs(b - 30.0 * S * 5 / 2e-3) < 1e-9 * b                       # all members over the slowest rank
        assert abs(alone - (4.0 + 6.0) * S * 5 / 3e-3) < 1e-9 * alone         # each rank's own sample, summed
        assert dev == 2e-8                                                    # the worst rank's deviation
    s0, s1 = res[0][3], res[1][3]
    assert set(s0).isdisjoint(s1) and sorted(s0 + s1) == list(range(8))


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.init_dist(1) is None
    assert bench.max_over_ranks(3.5) == 3.5 and bench.sum_over_ranks(2.0) == 2.0
