"""Seeded synthetic problems with the shapes of the benchmark configurations.

The reference publishes no dataset; each configuration is generated here from
its description (mesh, bathymetry, initial state, solver switches), seeded so
that every run and every test sees the same numbers.

  periodic_bump   N=3, 16x16 periodic Cartesian on [0,2]^2, b=0.1 sin(pi x)cos(pi y),
                  h = 1-b+0.05 exp(-50 r^2)                      (100 LS-RK4 steps, CFL 0.4)
  curved_lake     N=4, curved 512x512 on [0,1]^2 (x+0.03 sin sin), walls, 8 seeded
                  Gaussian bumps, lake at rest + seeded ripple   (1000 steps)
  dam_break       N=4, curved 256x256, b=0, circular dam of radius U[0.2,0.35], AV on
  tsunami_member  N=3, one ensemble member on a 2000 km square with a shelf,
                  seamounts and an Okada-type uplift (see ensemble.py)
"""
from __future__ import annotations

import numpy as np

from .host import Params, Problem, make_problem, mesh_cartesian, mesh_mapped


def _state(h, hu=None, hv=None, K=None, n2=None):
    """Pack nodal h, hu, hv [K*n2] into q [K][3][n2]."""
    q = np.zeros((K, 3, n2))
    q[:, 0, :] = h.reshape(K, n2)
    if hu is not None:
        q[:, 1, :] = hu.reshape(K, n2)
    if hv is not None:
        q[:, 2, :] = hv.reshape(K, n2)
    return q.reshape(-1)


def periodic_bump(N=3, nel=16, NumFlux=2, ES=1, steps=100, CFL=0.4) -> Problem:
    p = Params(N=N, CFL=CFL, T=1.0e9, g_const=9.81, NumFlux=NumFlux, ES=ES, rkOrder=4, rkSSP=0, MaxSteps=steps)
    m = mesh_cartesian(N, 0.0, 2.0, 0.0, 2.0, nel, nel, True, True)
    x, y = m.x, m.y
    b = 0.1 * np.sin(np.pi * x) * np.cos(np.pi * y)
    h = 1.0 - b + 0.05 * np.exp(-50.0 * ((x - 1.0) ** 2 + (y - 1.0) ** 2))
    n2 = (N + 1) ** 2
    return make_problem(p, m, b, _state(h, K=m.K, n2=n2), {"name": "periodic_bump", "nel": nel})


def conv_test(N=3, nel=8, T=0.1, CFL=0.4, NumFlux=0, L=2.0) -> Problem:
    """The reference's convergence test (Testcase 1, src/SW2D.cpp:312-319 and
    :829-833): Cartesian mesh on [0, L]^2 with Dirichlet boundaries carrying
    the exact solution h = 8 + cos x sin y cos t - b, u = 1/2, v = 3/2 over
    b = 2 + sin(2 pi y)/2 + cos(2 pi x), with the matching source term."""
    p = Params(N=N, CFL=CFL, T=T, g_const=9.81, NumFlux=NumFlux, ES=1, rkOrder=4, rkSSP=0, Testcase=1)
    m = mesh_cartesian(N, 0.0, L, 0.0, L, nel, nel)
    x, y = m.x, m.y
    b = 2.0 + 0.5 * np.sin(2.0 * np.pi * y) + np.cos(2.0 * np.pi * x)
    h = 8.0 + np.cos(x) * np.sin(y) - b
    n2 = (N + 1) ** 2
    return make_problem(p, m, b, _state(h, 0.5 * h, 1.5 * h, K=m.K, n2=n2), {"name": "conv_test", "nel": nel})


def conv_exact(prob, t):
    """Exact state of conv_test at time t, [K][3][n2] flattened."""
    m = prob.mesh
    h = 8.0 + np.cos(m.x) * np.sin(m.y) * np.cos(t) - prob.b
    return _state(h, 0.5 * h, 1.5 * h, K=m.K, n2=(prob.params.N + 1) ** 2)


def gaussian_bumps(x, y, seed, count=8):
    rng = np.random.default_rng(seed)
    b = np.zeros_like(x)
    for _ in range(count):
        amp = rng.uniform(0.05, 0.3)
        w = rng.uniform(0.03, 0.1)
        cx, cy = rng.uniform(0.0, 1.0, size=2)
        b += amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (w * w))
    return b


def curved_lake(N=4, nel=512, seed=0, ripple=0.01, steps=1000, NumFlux=0, CFL=0.4, rotate_seed=0,
                curve_order=None) -> Problem:
    p = Params(N=N, CFL=CFL, T=1.0e9, g_const=9.81, NumFlux=NumFlux, ES=1, rkOrder=4, rkSSP=0, MaxSteps=steps)
    m = mesh_mapped(N, 0.0, 1.0, 0.0, 1.0, nel, nel, amp=0.03, curve_order=curve_order, rotate_seed=rotate_seed)
    x, y = m.x, m.y
    b = gaussian_bumps(x, y, seed)
    h = 1.0 - b
    if ripple:
        rng = np.random.default_rng(seed + 1000)
        cx, cy = rng.uniform(0.25, 0.75, size=2)
        w = rng.uniform(0.03, 0.08)
        h = h + ripple * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (w * w))
    n2 = (N + 1) ** 2
    return make_problem(p, m, b, _state(h, K=m.K, n2=n2),
                        {"name": "curved_lake", "nel": nel, "seed": seed, "ripple": ripple})


def dam_break(N=4, nel=256, seed=0, steps=2000, NumFlux=0, CFL=0.4, AV=1, eps0=None, sigma_min=None,
              sigma_max=None, PP=0, rotate_seed=0) -> Problem:
    rng = np.random.default_rng(seed)
    r0 = rng.uniform(0.2, 0.35)
    cx, cy = rng.uniform(0.5 - 0.1, 0.5 + 0.1, size=2)
    # eps0 is scaled like the reference's dam-break runs: O(h * lambda_max)
    p = Params(N=N, CFL=CFL, DFL=0.1, T=1.0e9, g_const=9.81, NumFlux=NumFlux, ES=1, rkOrder=4, rkSSP=0,
               ArtificialViscosity=AV, PositivityPreserving=PP, MaxSteps=steps,
               epsilon_0=0.01 if eps0 is None else eps0,
               sigma_min=-6.0 if sigma_min is None else sigma_min,
               sigma_max=-2.0 if sigma_max is None else sigma_max)
    m = mesh_mapped(N, 0.0, 1.0, 0.0, 1.0, nel, nel, amp=0.03, rotate_seed=rotate_seed)
    x, y = m.x, m.y
    b = np.zeros_like(x)
    h = np.where((x - cx) ** 2 + (y - cy) ** 2 < r0 * r0, 2.0, 1.0)
    n2 = (N + 1) ** 2
    return make_problem(p, m, b, _state(h, K=m.K, n2=n2),
                        {"name": "dam_break", "nel": nel, "seed": seed, "radius": r0, "centre": (cx, cy)})


def bore(N=4, nel=256, seed=0, steps=2000, NumFlux=0, CFL=0.4, AV=1, eps0=None, sigma_min=None, sigma_max=None,
         rotate_seed=0) -> Problem:
    """A straight bore on the curved unit square (walls, b = 0): depth h_L
    behind the front s = x cos(a) + y sin(a) = s0, h_R = 1 ahead at rest, and
    the flow behind moving with the Rankine-Hugoniot velocity of a bore
    running into still water, u_L = S (1 - h_R / h_L) with
    S = sqrt(g h_L (h_L + h_R) / (2 h_R)); h_L ~ U[1.1, 1.8], a ~ U[0, 2 pi),
    s0 chosen so that the front crosses the middle of the domain."""
    rng = np.random.default_rng(50_000 + seed)
    g = 9.81
    hL, hR = rng.uniform(1.1, 1.8), 1.0
    a = rng.uniform(0.0, 2.0 * np.pi)
    S = np.sqrt(g * hL * (hL + hR) / (2.0 * hR))
    uL = S * (1.0 - hR / hL)
    p = Params(N=N, CFL=CFL, DFL=0.1, T=1.0e9, g_const=g, NumFlux=NumFlux, ES=1, rkOrder=4, rkSSP=0,
               ArtificialViscosity=AV, MaxSteps=steps,
               epsilon_0=0.01 if eps0 is None else eps0,
               sigma_min=-6.0 if sigma_min is None else sigma_min,
               sigma_max=-2.0 if sigma_max is None else sigma_max)
    m = mesh_mapped(N, 0.0, 1.0, 0.0, 1.0, nel, nel, amp=0.03, rotate_seed=rotate_seed)
    x, y = m.x, m.y
    s = (x - 0.5) * np.cos(a) + (y - 0.5) * np.sin(a)
    s0 = rng.uniform(-0.3, -0.1)
    behind = s < s0
    h = np.where(behind, hL, hR)
    hu = np.where(behind, hL * uL * np.cos(a), 0.0)
    hv = np.where(behind, hL * uL * np.sin(a), 0.0)
    b = np.zeros_like(x)
    n2 = (N + 1) ** 2
    return make_problem(p, m, b, _state(h, hu, hv, K=m.K, n2=n2),
                        {"name": "bore", "nel": nel, "seed": seed, "hL": hL, "angle": a})


TSUNAMI_SIZES = (64, 96, 128, 192, 256)


def tsunami_member(seed, N=3, steps=500, sizes=TSUNAMI_SIZES, AV=1, L=2.0e6, NumFlux=0, CFL=0.4,
                   eps0=2.0e4, sigma_min=-7.0, sigma_max=-3.0) -> Problem:
    """One member of the seeded tsunami ensemble: a K x K Cartesian mesh
    (K drawn from `sizes`) on an L x L square (metres, walls), a shelf 4000 m
    deep offshore rising linearly to 50 m over the last 200 km, 0-5 Gaussian
    seamounts, and the Okada uplift of a fault drawn from the seed (length
    50-400 km, width 20-150 km, top depth 5-30 km, dip 5-30 deg, strike 0-360
    deg, slip 1-15 m, thrust rake 90 deg) added to the sea surface at rest."""
    from . import okada
    rng = np.random.default_rng(10_000 + seed)
    nel = int(rng.choice(sizes))
    p = Params(N=N, CFL=CFL, DFL=0.1, T=1.0e9, g_const=9.81, NumFlux=NumFlux, ES=1, rkOrder=4, rkSSP=0,
               ArtificialViscosity=AV, epsilon_0=eps0, sigma_min=sigma_min, sigma_max=sigma_max, MaxSteps=steps,
               PosPresTOL=1e-4)
    m = mesh_cartesian(N, 0.0, L, 0.0, L, nel, nel)
    x, y = m.x, m.y
    shelf0 = L - 200.0e3
    depth = np.where(x < shelf0, 4000.0, 4000.0 - (4000.0 - 50.0) * (x - shelf0) / 200.0e3)
    b = -depth
    for _ in range(int(rng.integers(0, 6))):
        hgt = rng.uniform(500.0, 3000.0)
        w = rng.uniform(20.0e3, 80.0e3)
        cx, cy = rng.uniform(0.1 * L, shelf0), rng.uniform(0.1 * L, 0.9 * L)
        b = b + hgt * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (w * w))
    b = np.minimum(b, -50.0)
    f = okada.Fault(x0=rng.uniform(0.2 * L, 0.7 * L), y0=rng.uniform(0.2 * L, 0.8 * L),
                    depth=rng.uniform(5.0e3, 30.0e3), length=rng.uniform(50.0e3, 400.0e3),
                    width=rng.uniform(20.0e3, 150.0e3), strike=rng.uniform(0.0, 360.0), rake=90.0,
                    dip=rng.uniform(5.0, 30.0), slip=rng.uniform(1.0, 15.0))
    eta = okada.uplift_cartesian(x, y, f)
    h = -b + eta
    n2 = (N + 1) ** 2
    return make_problem(p, m, b, _state(h, K=m.K, n2=n2),
                        {"name": "tsunami_member", "seed": seed, "nel": nel, "fault": vars(f),
                         "max_uplift": float(np.abs(eta).max())})
