"""ORACLE test infrastructure: inputs of the reference program's runs of the
benchmark workload, made with NumPy alone (no module of the engine, no
shared library of this repository is loaded).

The workload: N = 4 on NEL x NEL curved quads over [0, 1]^2, the unit square
pushed through x -> x + 0.03 sin(2 pi x) sin(2 pi y) (y likewise), walls,
8 seeded Gaussian bumps, the lake at rest plus a seeded ripple.

* `write_mapped_mesh` writes that mesh as an ISM-V2 file, the format the
  reference reads (src/Mesh.cpp:698-1503): every element side a boundary
  curve of order m sampled at the Chebyshev-Gauss-Lobatto points
  -cos(k pi / m), faces numbered by first appearance over elements and
  sides.  It writes the same bytes as the engine's own mesh writer
  (tests/test_reference_program_cpu.py compares them).
* `write_case` writes the bathymetry bumps and the ripple for the case hook
  of the reference program (oracle/ref_shim/bench_case.cpp): with
  ESDG_REF_CASE set, SW2D::InitB and SW2D::InitQ evaluate them at the
  reference's own node coordinates, and the reference computes every
  derived array (metric terms, B_x and B_y by SW2D::CalcBDerivatives,
  normals, element sizes) itself.
* `lake_params` are the input.dat parameters, with T chosen so that the
  time-driven loop (src/deviceclass.cpp:895-930) takes a given number of
  steps.
"""
from __future__ import annotations

import math
import types

import numpy as np

# Side s of an element runs from corner ENDS[s][0] to corner ENDS[s][1]
# (sides 0 bottom, 1 right, 2 top, 3 left; src/Mesh.cpp:1017-1032).
ENDS = ((0, 1), (1, 2), (3, 2), (0, 3))


def _mapxy(u, v, xL, Lx, yL, Ly, amp):
    s = np.sin(2.0 * np.pi * (u - xL) / Lx) * np.sin(2.0 * np.pi * (v - yL) / Ly)
    return u + amp * Lx * s, v + amp * Ly * s


def mapped_mesh(nel, m=4, amp=0.03, xL=0.0, xR=1.0, yL=0.0, yR=1.0):
    """Corner nodes, element corner lists, face records and side curves of
    the mapped structured mesh.  Returns a dict of arrays (0-based ids)."""
    Lx, Ly = xR - xL, yR - yL
    NX = NY = nel
    ii, jj = np.meshgrid(np.arange(NX + 1, dtype=np.float64), np.arange(NY + 1, dtype=np.float64))
    nx_, ny_ = _mapxy(xL + Lx * ii / NX, yL + Ly * jj / NY, xL, Lx, yL, Ly, amp)
    nodes_x, nodes_y = nx_.reshape(-1), ny_.reshape(-1)
    ex, ey = np.meshgrid(np.arange(NX), np.arange(NY))
    ex, ey = ex.reshape(-1), ey.reshape(-1)
    c0 = ey * (NX + 1) + ex
    corners = np.stack([c0, c0 + 1, c0 + NX + 2, c0 + NX + 1], axis=1)  # counter-clockwise
    K = NX * NY
    # face records in (element, side) order; a face takes its number at its
    # first appearance
    a = np.stack([corners[:, ENDS[s][0]] for s in range(4)], axis=1).reshape(-1)
    b = np.stack([corners[:, ENDS[s][1]] for s in range(4)], axis=1).reshape(-1)
    nn = len(nodes_x) + 1
    key = np.minimum(a, b).astype(np.int64) * nn + np.maximum(a, b)
    _, first, inv, cnt = np.unique(key, return_index=True, return_inverse=True, return_counts=True)
    if cnt.max() > 2:
        raise ValueError("non-manifold edge")
    U = len(first)
    fid_of_u = np.empty(U, dtype=np.int64)
    fid_of_u[np.argsort(first, kind="stable")] = np.arange(U)
    rec = np.arange(4 * K)
    fid = fid_of_u[inv]
    second = np.full(U, -1, dtype=np.int64)
    other = rec != first[inv]
    second[inv[other]] = rec[other]
    F = U
    edges = np.zeros((F, 7), dtype=np.int64)
    fr = np.empty(F, dtype=np.int64)
    fr[fid_of_u] = first
    sr = np.empty(F, dtype=np.int64)
    sr[fid_of_u] = second
    edges[:, 0] = a[fr]
    edges[:, 1] = b[fr]
    edges[:, 2] = fr // 4
    edges[:, 4] = fr % 4
    has2 = sr >= 0
    s2 = np.where(has2, sr, 0)
    edges[:, 3] = np.where(has2, s2 // 4, -1)
    edges[:, 5] = np.where(has2, s2 % 4, -1)
    edges[:, 6] = np.where(has2, (a[s2] == a[fr]).astype(np.int64), 1)
    # side curves: the analytic map along the straight pre-image of the
    # side, end points snapped onto the mapped corner nodes
    xc = np.array([-math.cos(k * math.pi / m) for k in range(m + 1)])
    t = 0.5 * (xc + 1.0)
    pi_ = (np.arange(len(nodes_x)) % (NX + 1)).astype(np.float64)
    pj_ = (np.arange(len(nodes_x)) // (NX + 1)).astype(np.float64)
    pu, pv = xL + Lx * pi_ / NX, yL + Ly * pj_ / NY
    curves = np.empty((K, 4, m + 1, 2))
    for s in range(4):
        ca, cb = corners[:, ENDS[s][0]], corners[:, ENDS[s][1]]
        ua, va, ub, vb = pu[ca], pv[ca], pu[cb], pv[cb]
        u = ua[:, None] + (ub - ua)[:, None] * t[None, :]
        v = va[:, None] + (vb - va)[:, None] * t[None, :]
        X, Y = _mapxy(u, v, xL, Lx, yL, Ly, amp)
        X[:, 0], Y[:, 0] = nodes_x[ca], nodes_y[ca]
        X[:, m], Y[:, m] = nodes_x[cb], nodes_y[cb]
        curves[:, s, :, 0] = X
        curves[:, s, :, 1] = Y
    return {"nodes_x": nodes_x, "nodes_y": nodes_y, "corners": corners, "edges": edges, "curves": curves,
            "K": K, "F": F, "m": m, "face_of_side": fid.reshape(K, 4)}


def _pairs(x, y):
    return "".join("%.17g %.17g\n" % p for p in zip(x.tolist(), y.tolist()))


def write_mapped_mesh(path, nel, m=4, amp=0.03):
    """The mapped mesh as an ISM-V2 file.  Returns (K, F)."""
    M = mapped_mesh(nel, m=m, amp=amp)
    K, F, corners, edges, curves = M["K"], M["F"], M["corners"], M["edges"], M["curves"]
    with open(path, "w") as f:
        f.write("ISM-V2\n%d %d %d %d\n" % (len(M["nodes_x"]), F, K, m))
        f.write(_pairs(M["nodes_x"], M["nodes_y"]))
        sr = np.where(edges[:, 3] < 0, 0, np.where(edges[:, 6] == 1, edges[:, 5] + 1, -(edges[:, 5] + 1)))
        rows = np.stack([edges[:, 0] + 1, edges[:, 1] + 1, edges[:, 2] + 1, edges[:, 3] + 1, edges[:, 4] + 1, sr], 1)
        f.write("".join("%d %d %d %d %d %d\n" % tuple(r) for r in rows.tolist()))
        pts = curves.reshape(K, 4 * (m + 1), 2)
        chunk = 4096
        for e0 in range(0, K, chunk):
            parts = []
            for e in range(e0, min(K, e0 + chunk)):
                c = corners[e]
                parts.append("%d %d %d %d\n1 1 1 1\n" % (c[0] + 1, c[1] + 1, c[2] + 1, c[3] + 1))
                parts.append(_pairs(pts[e, :, 0], pts[e, :, 1]))
                parts.append("--- --- --- ---\n")
            f.write("".join(parts))
    return K, F


def bumps(seed, count=8):
    """The 8 seeded Gaussian bumps (amplitude U[0.05, 0.3], width U[0.03, 0.1],
    centre U[0, 1]^2), drawn in the order the engine's generator draws them."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        amp = rng.uniform(0.05, 0.3)
        w = rng.uniform(0.03, 0.1)
        cx, cy = rng.uniform(0.0, 1.0, size=2)
        out.append((float(amp), float(w), float(cx), float(cy)))
    return out


def ripple(seed, amp=0.01):
    """The seeded Gaussian ripple: (amplitude, width, centre x, centre y)."""
    rng = np.random.default_rng(seed + 1000)
    cx, cy = rng.uniform(0.25, 0.75, size=2)
    w = rng.uniform(0.03, 0.08)
    return (float(amp), float(w), float(cx), float(cy))


def write_case(path, seed, ripple_amp=0.01):
    """The case file of oracle/ref_shim/bench_case.cpp: b = sum of the bumps,
    h = 1 - b + ripple, hu = hv = 0."""
    bs = bumps(seed)
    with open(path, "w") as f:
        f.write("%d\n" % len(bs))
        for amp, w, cx, cy in bs:
            f.write("%.17g %.17g %.17g %.17g\n" % (amp, w, cx, cy))
        f.write("%.17g %.17g %.17g %.17g\n" % ripple(seed, ripple_amp))


def case_state(x, y, seed, ripple_amp=0.01):
    """b and h of the case at points (x, y), in the hook's order of operations."""
    b = np.zeros_like(x)
    for amp, w, cx, cy in bumps(seed):
        b = b + amp * np.exp(-((x - cx) * (x - cx) + (y - cy) * (y - cy)) / (w * w))
    amp, w, cx, cy = ripple(seed, ripple_amp)
    h = 1.0 - b + amp * np.exp(-((x - cx) * (x - cx) + (y - cy) * (y - cy)) / (w * w))
    return b, h


def lgl_nodes(N):
    """Legendre-Gauss-Lobatto nodes on [-1, 1] (Newton on (1 - x^2) P_N'(x))."""
    if N == 1:
        return np.array([-1.0, 1.0])
    x = -np.cos(np.pi * np.arange(N + 1) / N)
    for _ in range(100):
        P = np.zeros((N + 1, N + 1))
        P[:, 0], P[:, 1] = 1.0, x
        for k in range(2, N + 1):
            P[:, k] = ((2 * k - 1) * x * P[:, k - 1] - (k - 1) * P[:, k - 2]) / k
        dx = (x * P[:, N] - P[:, N - 1]) / ((N + 1) * P[:, N])
        x = x - dx
        if np.abs(dx).max() < 1e-15:
            break
    return x


def lake_params(nel, N, steps, seed=0, CFL=0.4, g=9.81, ripple_amp=0.01):
    """input.dat parameters of the workload with T set for `steps` time steps.

    The loop runs while t < T with dt = min(T - t, minEleSize/(N+1) CFL /
    lambda_max) (src/deviceclass.cpp:895-930).  T is (steps - 1/2) first
    steps: minEleSize is the square root of the smallest element area (the
    mapping's Jacobian 1 + 2 pi a sin(2 pi (x + y)) integrated over the
    element), lambda_max = max sqrt(g h) of the initial state at rest at the
    LGL nodes of the mapped elements.  Both are estimates good to far better
    than 1/(2 steps); the caller checks the number of steps the program
    reports."""
    amp = 0.03
    # smallest element area: the Jacobian at 6x6 Gauss points of every element
    gx, gw = np.polynomial.legendre.leggauss(6)
    h = 1.0 / nel
    e = (np.arange(nel) + 0.5) * h
    ex = e[:, None] + 0.5 * h * gx[None, :]  # [nel][6]
    # J(x, y) depends on x + y only
    area = np.full((nel, nel), 0.0)
    for a_ in range(6):
        for b_ in range(6):
            xs = ex[:, a_][:, None]
            ys = ex[:, b_][None, :]
            J = 1.0 + 2.0 * np.pi * amp * np.sin(2.0 * np.pi * (xs + ys))
            area += gw[a_] * gw[b_] * J
    area *= 0.25 * h * h
    min_ele = float(np.sqrt(area.min()))
    xl = lgl_nodes(N)
    u = (np.arange(nel)[:, None] + 0.5 * (xl[None, :] + 1.0)) / nel
    U, V = np.meshgrid(u.reshape(-1), u.reshape(-1))
    X, Y = _mapxy(U, V, 0.0, 1.0, 0.0, 1.0, amp)
    _, hh = case_state(X, Y, seed, ripple_amp)
    lam = float(np.sqrt(g * hh).max())
    dt = min_ele / (N + 1) * CFL / lam
    return types.SimpleNamespace(
        N=N, CFL=CFL, DFL=0.1, T=(steps - 0.5) * dt, g_const=g, ArtificialViscosity=0, PositivityPreserving=0,
        PosPresTOL=1e-4, epsilon_0=0.1, sigma_min=-16.0, sigma_max=-12.0, Testcase=0, ES=1, NumFlux=0,
        FluxDifferencing=1, rkOrder=4, rkSSP=0, NEpad=4, NEsurfpad=16, Nedgepad=16, NavgPad=10, DiscBottom=0,
        PartialDryTreatment=0, MaxSteps=0, ArrivalTimings=0, maximumElevation=0, h_0=0.0)
