"""Trains the learned troubled-cell indicator on the GPU.

    python -m esdgsem_mpiocca_b200.train_indicator --N 4 --out esdgsem_mpiocca_b200/weights/indicator_N4.npz

Training data are element snapshots of plain-solver runs with the modal
shock sensor on (the engine's reference-equivalent artificial-viscosity
path): seeded circular dam breaks and straight bores on the curved unit
square (and, at N = 3, tsunami scenarios of the ensemble generator with
seeds 100000 and up, disjoint from the benchmark's 0..255).  Every few
steps the engine's feature kernel labels each element with the sensor's
sigma; elements with sigma > -10 are all kept, the rest sampled at 5 %.
The network is then trained by the library's own BF16 forward/backward
kernels with Adam on FP32 master weights, and the decision margin is the
smallest one whose confident-but-wrong rate on held-out rows stays below
1e-4 for the sensor thresholds of both benchmark configurations.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import problems
from .deviceclass import Solver
from .indicator import DeviceMLP, IndicatorNet

# (sigma_min, sigma_max) of the dam-break and tsunami configurations
BANDS = ((-6.0, -2.0), (-7.0, -3.0))


def _runs(N, nruns):
    out = []
    for r in range(nruns):
        kind = r % 4
        if N == 3 and kind == 3:
            out.append(("tsunami", lambda r=r: problems.tsunami_member(100_000 + r, N=3, sizes=(64, 96, 128))))
        elif kind == 2:
            out.append(("bore", lambda r=r: problems.bore(N=N, nel=(128, 192)[r % 2], seed=r)))
        else:
            out.append(("dam_break", lambda r=r: problems.dam_break(N=N, nel=(128, 192, 256)[r % 3], seed=r)))
    return out


def collect(N, nruns, steps, every, max_rows, device, log):
    import torch
    ngl = N + 1
    mlp = DeviceMLP(IndicatorNet.fresh(ngl), device)
    Xs, ts, ss = [], [], []
    gen = torch.Generator(device=mlp.dev)
    gen.manual_seed(1234)
    total = 0
    snaps = 0
    for r, (kind, make) in enumerate(_runs(N, nruns)):
        prob = make()
        nsteps = steps if kind != "tsunami" else min(steps, 500)
        sol = Solver(prob, device_id=device)
        sol.run(max_steps=every)
        qp, bp, vp = sol.dc.state_pointers()
        done = every
        while True:
            X, t, s = mlp.features(qp, bp, vp, prob.K)
            sigma = t + s
            keep = torch.isfinite(t) & ((sigma > -10.0) | (torch.rand(prob.K, generator=gen, device=mlp.dev) < 0.05))
            Xs.append(X[keep])
            ts.append(t[keep])
            ss.append(s[keep])
            total += int(keep.sum())
            snaps += 1
            if done >= nsteps:
                break
            sol.dc.advance(every, 1.0e9)
            done += every
        torch.cuda.synchronize(mlp.dev)
        sol.close()
        log(f"run {r:3d} {kind:9s} K={prob.K:6d} steps={done:5d} rows so far {total}")
    X = torch.cat(Xs)
    t = torch.cat(ts)
    s = torch.cat(ss)
    if X.shape[0] > max_rows:
        idx = torch.randperm(X.shape[0], generator=gen, device=mlp.dev)[:max_rows]
        X, t, s = X[idx], t[idx], s[idx]
    return X, t, s, {"runs": nruns, "snapshots": snaps, "rows_kept": int(total), "rows_used": int(X.shape[0])}


def margin_table(y, t, s):
    """Confident-but-wrong rate of the decision rule for several margins."""
    sig_hat = (y + s).double()
    sig = (t + s).double()
    table = {}
    for m in (0.1, 0.25, 0.5, 0.75, 1.0, 1.5, 2.0):
        worst = 0.0
        for lo, hi in BANDS:
            zero_hat = sig_hat < lo - m
            full_hat = sig_hat > hi + m
            wrong = (zero_hat & (sig > lo)) | (full_hat & (sig < hi))
            worst = max(worst, float(wrong.double().mean()))
        fallback = max(float(((sig_hat >= lo - m) & (sig_hat <= hi + m)).double().mean()) for lo, hi in BANDS)
        table[str(m)] = {"confident_wrong": worst, "fallback": fallback}
    return table


def train(N, out, nruns=64, steps=1200, every=40, max_rows=10_000_000, iters=40_000, batch=16384, lr=2e-3,
          device=0, seed=0):
    import torch
    t0 = time.time()

    def log(msg):
        print(f"[{time.time() - t0:7.1f}s] {msg}", flush=True)

    torch.cuda.set_device(device)
    X, t, s, info = collect(N, nruns, steps, every, max_rows, device, log)
    M = X.shape[0]
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    perm = torch.randperm(M, generator=g, device=X.device)
    nval = max(M // 20, 1)
    Xv, tv, sv = X[perm[:nval]], t[perm[:nval]], s[perm[:nval]]
    Xt, tt = X[perm[nval:]], t[perm[nval:]]
    Mt = Xt.shape[0]
    mlp = DeviceMLP(IndicatorNet.fresh(N + 1, seed), device, blocks=64)
    log(f"training on {Mt} rows, validating on {nval}")
    hist = []
    order = torch.randperm(Mt, generator=g, device=X.device)
    pos = 0
    for it in range(1, iters + 1):
        if pos + batch > Mt:
            order = torch.randperm(Mt, generator=g, device=X.device)
            pos = 0
        idx = order[pos:pos + batch]
        pos += batch
        frac = it / iters
        cur = 1e-5 + 0.5 * (lr - 1e-5) * (1 + math.cos(math.pi * frac))
        if it <= 500:
            cur *= it / 500
        sse = mlp.train_step(Xt[idx].contiguous(), tt[idx].contiguous(), cur)
        if it % 2000 == 0 or it == iters:
            yv = mlp.forward(Xv)
            rmse = float(torch.sqrt(((yv - tv) ** 2).mean()))
            hist.append({"iter": it, "train_mse": float(sse) / batch, "val_rmse": rmse})
            log(f"iter {it:6d} lr {cur:.2e} train mse {float(sse) / batch:.4f} val rmse {rmse:.4f}")
    yv = mlp.forward(Xv)
    err = (yv - tv).abs()
    table = margin_table(yv, tv, sv)
    margin = next((float(m) for m, v in table.items() if v["confident_wrong"] <= 1e-4), 2.0)
    q = torch.quantile(err[:1_000_000].double(), torch.tensor([0.5, 0.9, 0.99, 0.999], dtype=torch.float64,
                                                               device=err.device)).tolist()
    meta = dict(info, N=N, iters=iters, batch=batch, lr=lr, seed=seed, train_rows=Mt, val_rows=nval,
                val_rmse=float(torch.sqrt(((yv - tv) ** 2).mean())), val_abs_err_quantiles=dict(
                    zip(("p50", "p90", "p99", "p999"), q)), margins=table, history=hist,
                seconds=time.time() - t0, bands=BANDS)
    net = mlp.to_net(**meta)
    net.margin = margin
    net.save(out)
    log(f"saved {out}: margin {margin}, val rmse {meta['val_rmse']:.4f}")
    return net


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=4)
    ap.add_argument("--out", required=True)
    ap.add_argument("--runs", type=int, default=64)
    ap.add_argument("--steps", type=int, default=1200)
    ap.add_argument("--every", type=int, default=40)
    ap.add_argument("--iters", type=int, default=40_000)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--max-rows", type=int, default=10_000_000)
    ap.add_argument("--summary", default=None)
    a = ap.parse_args()
    net = train(a.N, a.out, a.runs, a.steps, a.every, a.max_rows, a.iters, a.batch)
    if a.summary:
        with open(a.summary, "w") as f:
            json.dump(dict(net.meta, margin=net.margin), f, indent=1)


if __name__ == "__main__":
    main()
