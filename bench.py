#!/usr/bin/env python
"""Benchmark: DOF-stage updates/s of the plain FP64 ES-DGSEM step on B200.

Workload (the configuration the headline metric is quoted on): N=4 (5x5 LGL
nodes) on 512x512 curved quads over [0,1]^2 mapped by x+0.03 sin(2 pi x)
sin(2 pi y), reflecting walls, 8 seeded Gaussian bumps, lake at rest plus a
seeded ripple, 5-stage 4th-order low-storage RK at CFL 0.4.  A step is one
full time step (5 RK stages) over all 6,553,600 nodes; one DOF-stage update
is one RK stage applied to one node's (h, hu, hv).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (under torchrun) every rank advances its own replica of the
workload (the plain path has no data-path exchange on one mesh per GPU);
value is the sum over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF-stage updates/s on 1 B200: plain FP64 vs batched+learned at equal L2 error"
UNIT = "DOF-stage updates/s"
NEL, N_POLY, STAGES = 512, 4, 5
# compulsory traffic of the element kernel per node and stage: q in (24 B),
# Jinv, Y_xi, Y_eta, X_xi, X_eta, Bx, By (56 B), gRK in+out (48 B), q out (24 B)
ELEM_BYTES_PER_NODE = 152
# compulsory traffic of the whole stage (the above + face data once)
STAGE_BYTES_PER_NODE = 168


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# element-kernel variants of the engine at N = 4 (index = variant number)
ELEMENT_KERNELS_N4 = ("k_element_tma<5,2,2>", "k_element_tma<5,3,2>", "k_element_tma<5,2,3>",
                      "k_element_rows<5,30,2,1>", "k_element_rows<5,14,2,2>", "k_element_pair<5,3>",
                      "k_element_pair<5,4>")


def element_kernel_name(dc):
    ev = dc.element_variants()
    if not ev or ev["chosen"] < 0:
        return "k_element<5>"
    return ELEMENT_KERNELS_N4[ev["chosen"]]


def max_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(work: float, ms: float, dist=None, device: str = "cuda") -> float:
    """Whole-job rate of weakly scaled ranks: the work of all ranks over the
    slowest rank's time (ms)."""
    return sum_over_ranks(work, dist, device) / (max_over_ranks(ms, dist, device) / 1e3)


def ensemble_summary(dofs: float, ms: float, steps: int, alone_dofs: float, alone_ms: float, dev: float,
                     dist=None, device: str = "cuda"):
    """The ensemble line's rank aggregation: the batched rate of all ranks'
    members over the slowest rank's timed steps, the one-at-a-time rate as
    the sum of the ranks' own rates (each GPU solves its sample alone), and
    the largest deviation of any rank."""
    rate = job_rate(dofs * STAGES * steps, ms, dist, device)
    alone = sum_over_ranks(alone_dofs * STAGES * steps / (alone_ms / 1e3), dist, device)
    return rate, alone, max_over_ranks(dev, dist, device)


def member_seeds(rank: int, members: int) -> list:
    """Ensemble members of one rank: disjoint seed ranges, no exchange."""
    return list(range(rank * members, (rank + 1) * members))


def init_dist(ws: int, backend: str = "nccl"):
    """The process group for ws > 1 ranks (short timeout), else None."""
    if ws <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons while timing.

    Samples every `interval_ms`.  When the caller sets `window` (host times
    bracketing the timed region, device work included) only the samples
    taken inside it are kept; `in_window` counts them (a region of a few
    tens of milliseconds holds one or two)."""

    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, interval_ms: int = 200):
        self.gpu = gpu_index
        self.interval = interval_ms
        self.proc = None
        self.window = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.interval)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    @staticmethod
    def _stamp(text):
        try:
            return datetime.datetime.strptime(text.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def __exit__(self, *a):
        self.result = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.proc is None:
            return False
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        rows = []
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((self._stamp(f[0]), float(f[1]), float(f[2]), float(f[3]), f[5:9]))
            except ValueError:
                continue
        if self.window is not None:
            t0, t1 = self.window
            inside = [r for r in rows if r[0] is not None and t0 <= r[0] <= t1]
            self.result["in_window"] = len(inside)
            # a region shorter than the interval: the sample nearest to it
            if not inside and rows:
                mid = 0.5 * (t0 + t1)
                inside = [min((r for r in rows if r[0] is not None), key=lambda r: abs(r[0] - mid),
                              default=rows[-1])]
            rows = inside
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = {nm for r in rows for nm, v in zip(names, r[4]) if v.lower() == "active"}
        if rows:
            self.result.update({"sm_mhz": statistics.median(r[1] for r in rows),
                                "sm_max_mhz": max(r[2] for r in rows), "reasons": sorted(reasons),
                                "power_w": statistics.median(r[3] for r in rows), "samples": len(rows)})
        return False


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel):
    """DRAM bytes per launch of the element-kernel variant in use on this
    workload, from the committed ncu summary whose title names that exact
    variant (profiles/<kernel>_curved_lake_512_N4.md); None when no capture
    of that variant is committed."""
    import glob
    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", "k_element*_curved_lake_512_N4.md"))):
        with open(p) as f:
            lines = f.read().splitlines()
        if not lines or not lines[0].startswith("# ") or lines[0][2:].split(" ")[0] != kernel:
            continue
        for line in lines:
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1].strip())
    return None


def build_problem(seed=0):
    from esdgsem_mpiocca_b200 import problems
    return problems.curved_lake(N=N_POLY, nel=NEL, seed=seed, ripple=0.01, steps=0)


def workload_config(extra=None):
    """The workload's description, the same for both arms (no engine call:
    the sizes follow from the mesh generator's counts)."""
    K = NEL * NEL
    c = {"workload": "curved_lake: N=4, 512x512 curved quads on [0,1]^2 (x+0.03 sin sin), walls, 8 seeded "
                     "Gaussian bumps, lake at rest + 0.01 ripple, LS-RK4 (5 stages), CFL 0.4, ES flux NumFlux=0",
         "elements": K, "faces": 2 * NEL * (NEL + 1), "nodes": K * (N_POLY + 1) ** 2, "stages_per_step": STAGES,
         "l2_policy": "inputs larger than L2 (q+gRK+geometry ~0.9 GB resident vs 126 MB L2), no flush",
         "parallelism": "replica per GPU"}
    if extra:
        c.update(extra)
    return c


def run_cpu_sample(prob, threads, seconds_target=15.0, max_steps=None):
    """Oracle (C restatement of the reference kernels, OpenMP) on the full mesh."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle.oracle import OracleProblem
    op = OracleProblem(prob)
    t0 = time.perf_counter()
    out = op.run(T=1e9, max_steps=1)  # one step to size the sample
    t1 = time.perf_counter() - t0
    n = max(1, int(seconds_target / max(t1, 1e-6)))
    if max_steps:
        n = min(n, max_steps)
    t0 = time.perf_counter()
    out = op.run(q=out["q"], T=1e9, max_steps=n)
    el = time.perf_counter() - t0
    return prob.dofs() * STAGES * out["steps"] / el, out["steps"], el


def reference_program_sample(threads, steps, warmup, seed=0):
    """The reference program itself (oracle/_ref/esdg_ref: its main.cpp and
    src/*.cpp compiled unmodified, its .okl kernels built for OpenMP by the
    OCCA stand-in) on the workload: the mesh written as an ISM-V2 file by
    NumPy (oracle/ref_inputs.py) and read by the reference's own reader, the
    bathymetry and initial state evaluated by the case hook at the
    reference's own nodes (oracle/ref_shim/bench_case.cpp), and everything
    derived from them (metric terms, B_x, B_y, element sizes, time steps)
    computed by the reference.  No module or library of the engine is
    loaded.  Its own timer around DGtimeloop (main.cpp:1009-1072), for a run
    of `warmup` and one of `warmup + steps` time steps: the difference times
    `steps` steps after `warmup` warm-up steps; the step counts are checked
    against the program's own count of FindLambdaMax calls (one per step)."""
    import shutil
    import tempfile
    from oracle import ref_inputs, run_ref
    d = tempfile.mkdtemp(prefix="esdg_ref_case_")
    try:
        mesh = os.path.join(d, "curved_lake.mesh")
        case = os.path.join(d, "case.txt")
        ref_inputs.write_mapped_mesh(mesh, NEL)
        ref_inputs.write_case(case, seed)
        env = {"ESDG_REF_CASE": case, "ESDG_REF_COUNT": "1"}
        times = []
        for n in (warmup, warmup + steps):
            t, out, _ = run_ref.run_timed(ref_inputs.lake_params(NEL, N_POLY, n, seed=seed), mesh, None,
                                          threads=threads, timeout=600, extra_env=env)
            ran = run_ref.kernel_calls(out).get("FindLambdaMax", -1)
            if ran != n:
                raise RuntimeError(f"reference program took {ran} time steps, {n} asked for")
            times.append(t)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    el = times[1] - times[0]
    if not el > 0:
        raise RuntimeError(f"reference timings not increasing: {times}")
    nodes = NEL * NEL * (N_POLY + 1) ** 2
    return nodes * STAGES * steps / el, steps, el


def cpu_reference(threads, steps, warmup, prob=None, port_seconds=15.0):
    """The CPU baseline: the reference program on the host's cores, or, where
    it cannot run, the oracle (the reference kernels and time loop restated
    in C; needs `prob`).  Returns (cpu_baseline dict, steps, seconds)."""
    try:
        rate, nst, el = reference_program_sample(threads, steps, warmup)
        return {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"the reference program (main.cpp and src/ compiled unmodified against an OCCA-v0 "
                          f"stand-in, its okl kernels built for OpenMP) on the same 512x512 N=4 workload, its "
                          f"inputs written by NumPy and its bathymetry and state set by a case hook at its own "
                          f"nodes: {nst} time steps after {warmup} warm-up steps ({el:.1f} s), timed by its own "
                          f"DGtimeloop timer (difference of a {warmup}- and a {warmup + nst}-step run)"}, nst, el
    except Exception as e:  # noqa: BLE001 -- reported in the line
        log(f"reference program unavailable, timing the C restatement: {e}")
        if prob is None:
            prob = build_problem(seed=0)
        rate, nst, el = run_cpu_sample(prob, threads, seconds_target=port_seconds, max_steps=steps)
        return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": f"{nst} full time steps of the same 512x512 N=4 workload ({el:.1f} s) with the C "
                          f"oracle (reference kernels and time loop restated), OpenMP",
                "reference_program_unavailable": str(e).splitlines()[0][:300] if str(e) else type(e).__name__}, \
            nst, el


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="leave the batched+learned ensemble comparison out of the default line")
    ap.add_argument("--ensemble-steps", type=int, default=100,
                    help="time steps of the ensemble comparison in the default line")
    ap.add_argument("--workload", default="curved_lake", choices=["curved_lake", "ensemble", "serving", "dambreak"],
                    help="curved_lake: the headline single-mesh workload; ensemble: 256 seeded tsunami "
                         "members batched vs one at a time; serving: Poisson request streams; dambreak: the "
                         "learned indicator against the plain sensor on the N=4 dam break")
    ap.add_argument("--rates", default="10,100,1000", help="serving workload: arrival rates (requests/s)")
    ap.add_argument("--requests", type=int, default=48, help="serving workload: requests per rate")
    ap.add_argument("--hbm-gb", type=float, default=40.0, help="serving workload: HBM given to the arenas")
    ap.add_argument("--max-live-nodes", type=float, default=4e6,
                    help="serving workload, shortest-job-first run: nodes in flight at most")
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--indicator-schedule", default="stage", choices=["stage", "step"],
                    help="ensemble workload: the learned indicator at every RK stage or once per step")
    ap.add_argument("--alone-members", type=int, default=15,
                    help="ensemble workload: members solved one at a time for the plain-path rate")
    ap.add_argument("--element-variant", type=int, default=-1,
                    help="curved_lake: fix the element-kernel variant (index into the engine's variant list; "
                         "-1: the autotuner picks), e.g. to profile one variant")
    args = ap.parse_args()
    if args.workload == "ensemble":
        return ensemble_bench(args)
    if args.workload == "serving":
        return serving_bench(args)
    if args.workload == "dambreak":
        return dambreak_bench(args)
    ws, rank, local = dist_env()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        return reference_arm(args, ws, rank)

    import torch
    torch.cuda.set_device(local)
    dist = init_dist(ws)

    from esdgsem_mpiocca_b200.deviceclass import Solver
    prob = build_problem(seed=rank)
    s = Solver(prob, device_id=local)
    stream = torch.cuda.Stream()
    s.dc.set_stream(stream.cuda_stream)
    if args.element_variant >= 0:
        s.dc.set_element_variant(args.element_variant)
    # warm-up: builds the step graph and runs W steps
    s.run(T=1e9, max_steps=args.warmup)
    torch.cuda.synchronize()

    # ---- device-timed region: inputs resident in HBM ----
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = s.dc.kernel_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local, 20) as ck:
        tw0 = time.time()
        with torch.cuda.stream(stream):
            e0.record(stream)
            t_sim, nsteps_done = s.dc.advance(args.steps, 1e9)
            e1.record(stream)
        torch.cuda.synchronize()
        ck.window = (tw0, time.time())
    if dist:
        dist.barrier()
    launches = s.dc.kernel_launches() - launches0
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, dist)
    value = job_rate(prob.dofs() * STAGES * args.steps, ms, dist)

    # ---- dominant kernel duration, timed live on the engine's stream ----
    kern = time_element_kernel(s, stream, prob)

    # ---- end to end through the C ABI with host buffers ----
    e2e = e2e_run(s, prob, stream, args.steps, dist, ws)

    hbm, peak_kind = peaks()
    ach = ELEM_BYTES_PER_NODE * prob.dofs() / (kern["ms"] / 1e3) / 1e9
    traffic = profiled_traffic(element_kernel_name(s.dc))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded curved_lake generator; no dataset exists)",
        "config": workload_config(),
        "sim_time_reached": t_sim,
        "roofline": {"bound": "hbm", "kernel": element_kernel_name(s.dc), "achieved": ach, "peak": hbm, "unit": "GB/s",
                     "frac": ach / hbm, "peak_kind": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
                     "traffic": traffic,
                     "bytes_per_node": ELEM_BYTES_PER_NODE, "launch_ms": kern["ms"],
                     "face_kernel_ms": kern["face_ms"],
                     "stage": {"bytes_per_node": STAGE_BYTES_PER_NODE,
                               "achieved": STAGE_BYTES_PER_NODE * prob.dofs() * STAGES * args.steps /
                               (ms_max / 1e3) / 1e9}},
        "e2e": e2e,
        "autotuned": s.dc.element_variants(),
        "gpu_launches": int(launches),
        "clocks": ck.result,
    }
    # ---- the same step loop for about a second, outside the timed region:
    # the clocks and power a sustained run settles at, and its step time ----
    nsus = max(args.steps, int(1000.0 / max(ms / args.steps, 0.05)))
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    with Clocks(local, 50) as ck2:
        with torch.cuda.stream(stream):
            e2.record(stream)
            s.dc.advance(nsus, 1e9)
            e3.record(stream)
        torch.cuda.synchronize()
    line["clocks_sustained"] = dict(ck2.result, steps=nsus, ms_per_step=e2.elapsed_time(e3) / nsus)
    s.close()
    # ---- the batched+learned half of the metric: the 256-member tsunami
    # ensemble, batched with the learned indicator vs one at a time plain ----
    if not args.no_ensemble:
        line["batched_learned"] = ensemble_measure(256, args.ensemble_steps, 3, 10, local, dist, ws, rank,
                                                   attribution=False, every_stage=True)
        line["batched_learned"]["workload"] = (
            "ensemble of 256 seeded tsunami members per GPU, N=3, K in {64..256}^2 on 2000 km squares, shelf, "
            "seamounts, Okada uplift, artificial viscosity; batched arena with the learned indicator (every RK "
            "stage, as the reference's sensor) and the active set vs 10 members (every size class) one at a "
            "time on the plain path; "
            f"{args.ensemble_steps} LS-RK4 steps after 3 warm-up steps (the configuration runs 500)")
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference(os.cpu_count() or 1, args.steps, args.warmup, prob=prob)[0]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def time_element_kernel(s, stream, prob, reps=10):
    """Average duration of the dominant kernel (k_element) and of the face
    kernel: real steps launched kernel by kernel with CUDA events recorded
    on the stream they are launched on (esdg_profile_steps)."""
    face_ms, elem_ms = s.dc.profile_steps(reps)
    return {"ms": elem_ms, "face_ms": face_ms}


def e2e_run(s, prob, stream, steps, dist, ws):
    """copyDeviceVariables(q) + DGtimeloop(steps) + o_q.copyTo(q), host
    buffers pinned, timed on the device around the three calls."""
    import torch
    qh = torch.from_numpy(prob.q0.copy()).pin_memory()
    qo = torch.empty_like(qh).pin_memory()
    qn, qon = qh.numpy(), qo.numpy()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0.record(stream)
        s.dc.copy_q_from_host(qn)
        t, n = s.run(T=1e9, max_steps=steps)
        s.dc.copy_q_to_host(qon)
        e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    assert np.isfinite(qon).all()
    work = sum_over_ranks(prob.dofs() * STAGES * steps, dist)
    return {"value": work / (ms / 1e3), "unit": UNIT,
            "h2d_bytes_per_step": qh.numel() * 8 / steps, "d2h_bytes_per_step": qo.numel() * 8 / steps,
            "calls": "esdg_copy_q_from_host + esdg_dg_timeloop + esdg_copy_q_to_host"}


def member_sizes(seeds):
    """(K, F) of each tsunami member without building it (the size is the
    first draw of the member's generator)."""
    from esdgsem_mpiocca_b200.problems import TSUNAMI_SIZES
    out = []
    for s in seeds:
        nel = int(np.random.default_rng(10_000 + s).choice(TSUNAMI_SIZES))
        out.append((nel * nel, 2 * nel * (nel + 1)))
    return out


def _alone_sample(seeds, k):
    """k members spread over the size classes (every class represented)."""
    from esdgsem_mpiocca_b200.problems import TSUNAMI_SIZES
    by = {n: [] for n in TSUNAMI_SIZES}
    for sd, (K, _) in zip(seeds, member_sizes(seeds)):
        by[int(round(K ** 0.5))].append(sd)
    out = []
    while len(out) < min(k, len(seeds)):
        for n in TSUNAMI_SIZES:
            if by[n] and len(out) < k:
                out.append(by[n].pop(0))
    return out


def ensemble_measure(members, steps, warm, alone_members, local, dist, ws, rank, attribution=True,
                     every_stage=False):
    """The ensemble configuration: seeded tsunami members (N=3, K in
    {64..256}^2 on 2000 km squares, artificial viscosity) advanced in one
    arena with the learned indicator and the active set, against the plain
    path -- a sample of the same members (every size class) solved one at a
    time by the single-mesh engine with the modal sensor and the viscous
    terms on every element (the reference's path).  Returns both rates,
    their ratio, the largest relative L2 deviation of a batched learned
    member from its plain solution after the same steps, the agreement of
    the learned and the modal viscosity flags on the plain solutions' final
    states, the indicator's decision shares, the clocks of the timed region
    and, with `attribution`, the batched rates of the other indicator modes.
    The learned indicator runs once per step (every_stage=False; its
    viscosity and active set kept for the step's stages) or at every stage.
    Per-step work: src/deviceclass.cpp:897-1130 for every member."""
    import torch
    from esdgsem_mpiocca_b200 import problems
    from esdgsem_mpiocca_b200.deviceclass import Solver
    from esdgsem_mpiocca_b200.ensemble import Ensemble
    from esdgsem_mpiocca_b200.indicator import IndicatorNet
    total = warm + steps
    seeds = member_seeds(rank, members)
    sizes = member_sizes(seeds)
    Kc, Fc = sum(k for k, _ in sizes), sum(f for _, f in sizes)
    p0 = problems.tsunami_member(seeds[0], steps=steps, sizes=(8,)).params  # parameters only
    net = IndicatorNet.default(3)
    sample = _alone_sample(seeds, alone_members)
    attr_steps = min(steps, 50)
    ens = Ensemble(3, len(seeds), Kc, Fc, NumFlux=p0.NumFlux, g_const=p0.g_const, PosPresTOL=p0.PosPresTOL,
                   ArtificialViscosity=p0.ArtificialViscosity, epsilon_0=p0.epsilon_0,
                   sigma_max=p0.sigma_max, sigma_min=p0.sigma_min, device_id=local)
    ens.set_indicator(2, net)
    ens.set_indicator_every_stage(every_stage)
    t0 = time.perf_counter()
    dofs, ids, kept = 0, {}, {}
    for sd in seeds:
        pr = problems.tsunami_member(sd)
        ids[sd] = ens.add(pr, T=1e9, max_steps=total + (3 * attr_steps if attribution else 0))
        dofs += pr.dofs()
        if sd in sample:
            kept[sd] = pr
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    ens.set_stream(stream.cuda_stream)
    all_dofs = sum_over_ranks(dofs, dist)

    def timed(nsteps):
        ens.indicator_stats(reset=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = ens.kernel_launches()
        with Clocks(local) as ck:
            with torch.cuda.stream(stream):
                e0.record(stream)
                ens.advance(nsteps)
                e1.record(stream)
            torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), dist)
        st = [ens.status(i) for i in ids.values()]
        return {"ms": ms, "rate": all_dofs * STAGES * nsteps / (ms / 1e3), "launches": ens.kernel_launches() - l0,
                "stats": ens.indicator_stats(), "clocks": ck.result, "steps": [x["steps"] for x in st],
                "errors": sum(1 for x in st if x["status"] != 0)}

    # batched, learned indicator with the active set: W untimed steps, then
    # the timed steps; the sampled members' states are kept for the
    # deviation check
    ens.advance(warm)
    learned = timed(steps)
    learned["all_done"] = all(x == total for x in learned["steps"])
    qb = {sd: ens.q(ids[sd]) for sd in sample}
    attrib = {}
    if attribution:  # the same arena continued with the other schedule and indicator modes
        ens.set_indicator_every_stage(not every_stage)
        attrib["other_schedule"] = timed(attr_steps)
        ens.set_indicator_every_stage(every_stage)
        for m in (0, 1):
            ens.set_indicator(m)
            attrib[m] = timed(attr_steps)
    ens.close()
    # one at a time, plain path (modal sensor, viscous terms everywhere)
    adofs, ams, dev, agree, nflag = 0, 0.0, 0.0, 0, 0
    for sd in sample:
        pr = kept[sd]
        s = Solver(pr, device_id=local)
        st = torch.cuda.Stream()
        s.dc.set_stream(st.cuda_stream)
        s.run(T=1e9, max_steps=warm)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(st):
            a0.record(st)
            s.dc.advance(steps, 1e9)
            a1.record(st)
        torch.cuda.synchronize()
        ams += a0.elapsed_time(a1)
        adofs += pr.dofs()
        qa = s.q().reshape(pr.K, 3, -1)
        qm = qb[sd].reshape(pr.K, 3, -1)
        for v in range(3):
            dev = max(dev, float(np.linalg.norm(qm[:, v] - qa[:, v]) / max(np.linalg.norm(qa[:, v]), 1e-300)))
        # flags of the two indicators on the plain solution's final state
        _, v0 = s.rhs()
        s.dc.set_indicator(2, net)
        _, v2 = s.rhs()
        agree += int(((v0 > 0) == (v2 > 0)).sum())
        nflag += int(v0.size)
        s.close()
    _, alone, dev = ensemble_summary(dofs, learned["ms"], steps, adofs, ams, dev, dist)
    stt = learned["stats"]
    decided = stt["net_zero"] + stt["net_full"]
    evals = decided + stt["modal"]
    out = {"value": learned["rate"], "unit": UNIT, "ms_per_step": learned["ms"] / steps, "steps": steps,
           "warmup": warm, "members": len(seeds) * ws, "nodes": all_dofs, "setup_s": setup_s,
           "all_done": learned["all_done"], "members_with_error": learned["errors"],
           "plain_one_at_a_time": {"value": alone, "unit": UNIT, "members": len(sample),
                                   "note": "modal sensor and viscous terms on every element (reference path)"},
           "ratio_batched_learned_over_plain": learned["rate"] / alone,
           "max_rel_l2_deviation_vs_plain": dev,
           "flag_agreement": agree / max(nflag, 1),
           "indicator": {"network_settled": decided / max(evals, 1), "modal_fallback": stt["modal"] / max(evals, 1),
                         "viscous_share": stt["viscous"] / max(evals, 1), "margin": net.margin,
                         "schedule": "every RK stage" if every_stage else "once per step (start of step)"},
           "gpu_launches": int(learned["launches"]), "clocks": learned["clocks"]}
    if attribution:
        out["attribution_batched"] = {"modal_full_path": attrib[0]["rate"], "modal_active_set": attrib[1]["rate"],
                                      "learned_active_set": learned["rate"],
                                      ("learned_every_stage" if not every_stage else "learned_once_per_step"):
                                          attrib["other_schedule"]["rate"],
                                      "steps": attr_steps}
    return out


def ensemble_bench(args):
    """The ensemble configuration alone (see ensemble_measure), as its own
    JSON line."""
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(ws)
    steps = args.steps if args.steps != 20 else 500
    warm = max(args.warmup, 3)
    r = ensemble_measure(args.members, steps, warm, args.alone_members, local, dist, ws, rank,
                         every_stage=args.indicator_schedule == "stage")
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": ws, "steps": steps,
            "warmup": warm, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (indicator network: bf16 weights, fp32 accumulation)",
            "data": "synthetic (seeded tsunami members: shelf, seamounts, Okada uplift)",
            "config": {"workload": f"ensemble of {r['members']} tsunami members, N=3, K in {{64..256}}^2 on 2000 km "
                                   f"squares, {steps} LS-RK4 steps each, artificial viscosity; batched arena with "
                                   "the learned indicator and the active set",
                       "members": r["members"], "nodes": r["nodes"], "setup_s": r["setup_s"],
                       "all_done": r["all_done"], "sharding": "members split across ranks, no exchange",
                       "members_with_error": r["members_with_error"],
                       "l2": "state (~16 GB at 256 members) far larger than L2",
                       "indicator_schedule": args.indicator_schedule}}
    for k in ("plain_one_at_a_time", "ratio_batched_learned_over_plain", "max_rel_l2_deviation_vs_plain",
              "flag_agreement", "indicator", "attribution_batched", "gpu_launches", "clocks"):
        line[k] = r[k]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def serving_bench(args):
    """The serving configuration: Poisson streams of tsunami solves (K from
    32^2 to 256^2, N in {3, 4}, 200-2000 steps) at several arrival rates,
    served by the continuous-batching server (learned indicator, active
    set) and, for the same streams, one request at a time by the plain
    single-mesh path.  Reports p50/p99 latency and throughput of both."""
    import torch
    from esdgsem_mpiocca_b200 import serving
    ws, rank, local = dist_env()
    if ws > 1:
        # latency percentiles are per server; the loop runs on one GPU
        if rank == 0:
            print(json.dumps({"metric": METRIC, "unavailable": "the serving workload runs on one GPU"}), flush=True)
        return 0
    torch.cuda.set_device(local)
    rates = [float(x) for x in args.rates.split(",")]
    t0 = time.perf_counter()
    streams = {rate: serving.make_requests(args.requests, rate, seed=1000 * rank + int(rate)) for rate in rates}
    setup_s = time.perf_counter() - t0
    srv = serving.Server(hbm_bytes=args.hbm_gb * 1e9, max_instances=256, device_id=local)
    # warm-up: one small request through each arena
    serving.serve(serving.make_requests(2, 1e6, seed=7, sizes=(32,), horizons=(5, 5)), srv, realtime=False)
    out = []
    with Clocks(local) as ck:
        for rate in rates:
            srv.max_live_nodes = None
            b = serving.serve(serving.fresh(streams[rate]), srv, realtime=True)
            srv.max_live_nodes = int(args.max_live_nodes)
            j = serving.serve(serving.fresh(streams[rate]), srv, realtime=True, policy="sjf")
            srv.max_live_nodes = None
            a = serving.serve_one_at_a_time(serving.fresh(streams[rate]), indicator=0, device_id=local)
            out.append({"rate_per_s": rate, "batched": b, "batched_sjf_capped": j, "plain_one_at_a_time": a,
                        "throughput_ratio": b["throughput_dof_stages_per_s"] / a["throughput_dof_stages_per_s"],
                        "p99_ratio": a["p99_s"] / b["p99_s"],
                        "sjf_p50_ratio": a["p50_s"] / j["p50_s"], "sjf_p99_ratio": a["p99_s"] / j["p99_s"],
                        "sjf_throughput_ratio": j["throughput_dof_stages_per_s"] / a["throughput_dof_stages_per_s"]})
        srv.close()
        # the same server architecture with the exact modal active set
        srv1 = serving.Server(hbm_bytes=args.hbm_gb * 1e9, max_instances=256, device_id=local, indicator=1)
        serving.serve(serving.make_requests(2, 1e6, seed=7, sizes=(32,), horizons=(5, 5)), srv1, realtime=False)
        m1 = serving.serve(serving.fresh(streams[rates[-1]]), srv1, realtime=True)
        srv1.close()
    top = out[-1]["batched"]
    line = {"metric": METRIC, "value": top["throughput_dof_stages_per_s"], "unit": UNIT, "n_gpus": 1,
            "steps": None, "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 (indicator network: bf16 weights, fp32 accumulation)",
            "data": "synthetic (seeded tsunami requests, Poisson arrivals)",
            "config": {"workload": f"serving: {args.requests} requests per rate, K in 32^2..256^2, N in {{3,4}}, "
                                   "200-2000 steps, continuous batching with admission by HBM footprint "
                                   f"({args.hbm_gb} GB of arenas), learned indicator + active set; FIFO, and "
                                   f"shortest job first with at most {args.max_live_nodes:.0f} nodes in flight",
                       "setup_s": setup_s, "value_is": f"batched throughput at {rates[-1]} requests/s"},
            "rates": out, "batched_modal_active_set_at_top_rate": m1, "clocks": ck.result}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def dambreak_bench(args):
    """The learned-indicator configuration: circular dam break, N=4 on 256^2
    curved quads, flat bottom, artificial viscosity, 2000 steps; the plain
    path (modal sensor, viscous terms everywhere), the exact modal active set
    and the learned indicator from the same initial state.  Reports their
    rates, the learned run's deviation from the plain run (relative L2 per
    variable) and the flag agreement of the two indicators on the plain
    run's states."""
    import torch
    from esdgsem_mpiocca_b200 import problems
    from esdgsem_mpiocca_b200.deviceclass import Solver
    from esdgsem_mpiocca_b200.indicator import IndicatorNet
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    steps = args.steps if args.steps != 20 else 2000
    warm = max(args.warmup, 3)
    prob = problems.dam_break(N=4, nel=256, seed=rank, steps=steps + warm)
    net = IndicatorNet.default(4)
    stream = torch.cuda.Stream()
    runs = {}
    with Clocks(local) as ck:
        for mode in (0, 1, 2):
            s = Solver(prob, device_id=local, indicator=mode, net=net if mode == 2 else None)
            s.dc.set_stream(stream.cuda_stream)
            s.run(T=1e9, max_steps=warm)
            if mode:
                s.dc.indicator_stats(reset=True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            with torch.cuda.stream(stream):
                e0.record(stream)
                s.dc.advance(steps, 1e9)
                e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            runs[mode] = {"ms": ms, "rate": prob.dofs() * STAGES * steps / (ms / 1e3), "q": s.q(),
                          "stats": s.dc.indicator_stats() if mode else None}
            s.close()
    K, n2 = prob.K, prob.ngl ** 2
    q0 = runs[0]["q"].reshape(K, 3, n2)
    dev = {}
    for mode in (1, 2):
        qm = runs[mode]["q"].reshape(K, 3, n2)
        dev[mode] = [float(np.linalg.norm(qm[:, v] - q0[:, v]) / np.linalg.norm(q0[:, v])) for v in range(3)]
    # flag agreement on the plain run's final state
    s0 = Solver(prob, device_id=local, q0=runs[0]["q"])
    _, v0 = s0.rhs()
    s0.close()
    s2 = Solver(prob, device_id=local, q0=runs[0]["q"], indicator=2, net=net)
    _, v2 = s2.rhs()
    s2.close()
    st = runs[2]["stats"]
    ev = st["net_zero"] + st["net_full"] + st["modal"]
    line = {"metric": METRIC, "value": runs[2]["rate"], "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": warm,
            "ms_per_step": runs[2]["ms"] / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (indicator network: bf16 weights, fp32 accumulation)",
            "data": "synthetic (seeded circular dam break)",
            "config": {"workload": f"dam break: N=4, 256x256 curved quads, b=0, artificial viscosity, {steps} steps; "
                                   "learned indicator + active set", "nodes": prob.dofs(),
                       "radius": prob.meta["radius"]},
            "plain_modal_full_path": runs[0]["rate"], "modal_active_set": runs[1]["rate"],
            "ratio_learned_over_plain": runs[2]["rate"] / runs[0]["rate"],
            "rel_l2_deviation_learned_vs_plain": dev[2], "rel_l2_deviation_active_set_vs_plain": dev[1],
            "flag_agreement_final_state": float(((v0 > 0) == (v2 > 0)).mean()),
            "viscosity_identical_final_state": float((v0 == v2).mean()),
            "network_settled": (st["net_zero"] + st["net_full"]) / max(ev, 1),
            "viscous_share": st["viscous"] / max(ev, 1), "clocks": ck.result}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def reference_arm(args, ws, rank):
    """The reference's CPU path for this workload, on the host's cores: the
    reference program with the --steps and --warmup counts.  Nothing
    of the engine is imported or loaded in this process."""
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    cb, nst, el = cpu_reference(threads, args.steps, args.warmup, port_seconds=30.0)
    rate = cb["value"]
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": ws, "steps": nst, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / nst, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded curved_lake generator; no dataset exists)", "impl": "reference",
            "config": workload_config(), "cpu_baseline": cb,
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main() or 0)
