"""ORACLE -- test infrastructure only.

NumPy restatement of the learned indicator's arithmetic (the engine's
esdgsem_mpiocca_b200/csrc/esdg_mlp.cuh): element features, the modal
sensor value sigma (okl/ShockCapturing/ShockCapturing.okl:131-204), the
network's forward pass with the same BF16 roundings as the tensor-core
kernels (X, W1, W2 and the first activation rounded to BF16, everything
else in float64 here), its exact gradient, and one Adam step.  Imported only
by tests/.
"""
from __future__ import annotations

import numpy as np

H = 32
S_MIN = -12.0


def bf16(a):
    """Round float32 values to BF16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    nan = np.isnan(a)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(nan, a, out)


def nin(ngl):
    return 3 * ngl * ngl + 3


def kp(ngl):
    return (nin(ngl) + 15) // 16 * 16


def layout(ngl):
    k = kp(ngl)
    L = {"kp": k, "w1": 0}
    L["b1"] = L["w1"] + H * k
    L["w2"] = L["b1"] + H
    L["b2"] = L["w2"] + H * H
    L["w3"] = L["b2"] + H
    L["b3"] = L["w3"] + H
    L["total"] = (L["b3"] + 1 + 3) // 4 * 4
    return L


def unpack(P, ngl):
    L = layout(ngl)
    k = L["kp"]
    return (P[L["w1"]:L["b1"]].reshape(H, k), P[L["b1"]:L["w2"]], P[L["w2"]:L["b2"]].reshape(H, H),
            P[L["b2"]:L["w3"]], P[L["w3"]:L["b3"]], P[L["b3"]])


def sensor_sigma(eta, V, ZeroTOL=1e-5, tiny_out=None):
    """sigma per element: eta [K][n*n] (node (xi, eta) at eta*n + xi), V = VdmInv [n][n].
    tiny_out (optional list) receives the mask n1 < ZeroTOL."""
    n = V.shape[0]
    N = n - 1
    m = eta.reshape(-1, n, n)                   # [k][row = eta index][col = xi index]
    M1 = np.einsum("il,kjl->kij", V, m)         # M1[i][j] = sum_l V[i][l] m[j][l]
    w = np.einsum("kil,jl->kij", M1, V)         # w[i][j] = sum_l M1[i][l] V[j][l]
    z1 = (w[:, :N, N] ** 2).sum(1) + (w[:, N, :N] ** 2).sum(1) + w[:, N, N] ** 2
    z2 = (w[:, :N - 1, N - 1] ** 2).sum(1) + (w[:, N - 1, :N - 1] ** 2).sum(1) + w[:, N - 1, N - 1] ** 2
    n1 = (w ** 2).sum((1, 2))
    n2s = (w[:, :N, :N] ** 2).sum((1, 2))
    with np.errstate(divide="ignore", invalid="ignore"):
        t1 = np.where(n1 < ZeroTOL, 0.0, z1 / n1)
        t2 = np.where(n1 < ZeroTOL, 0.0, z2 / n2s)
        if tiny_out is not None:
            tiny_out.append(n1 < ZeroTOL)
        return np.log10(np.maximum(t1, t2))


def _stats(v):
    mean = v.mean(1)
    d = v - mean[:, None]
    rms = np.sqrt((d * d).mean(1))
    tot = mean * mean + rms * rms
    with np.errstate(divide="ignore", invalid="ignore"):
        s = np.where((tot > 0) & (rms > 0), np.maximum(np.log10(rms * rms / tot), S_MIN), S_MIN)
        flat = ~((rms > 1e-12 * np.abs(mean)) & (rms > 0))
        x = np.where(flat[:, None], 0.0, d / rms[:, None])
    return x, s


def features(q, b, ngl):
    """Feature rows X [K][kp] (BF16 values as float32) and s_eta [K]."""
    n2 = ngl * ngl
    q = np.asarray(q, dtype=np.float64).reshape(-1, 3, n2)
    K = q.shape[0]
    eta = q[:, 0, :] + np.asarray(b, dtype=np.float64).reshape(K, n2)
    X = np.zeros((K, kp(ngl)), dtype=np.float32)
    s_eta = None
    for f, v in enumerate((eta, q[:, 1, :], q[:, 2, :])):
        x, s = _stats(v)
        X[:, f * n2:(f + 1) * n2] = x
        X[:, 3 * n2 + f] = 0.25 * s
        if f == 0:
            s_eta = s
    return bf16(X), s_eta


def target(q, b, V, ngl, ZeroTOL=1e-5):
    """clamp(sigma, -12, 0) - s_eta; NaN where the modal energy is below ZeroTOL."""
    n2 = ngl * ngl
    q = np.asarray(q, dtype=np.float64).reshape(-1, 3, n2)
    eta = np.asarray(b, dtype=np.float64).reshape(-1, n2) + q[:, 0, :]
    tiny = []
    sg = sensor_sigma(eta, V, ZeroTOL, tiny)
    _, s_eta = features(q, b, ngl)
    t = np.clip(np.nan_to_num(sg, neginf=S_MIN), S_MIN, 0.0) - s_eta
    return np.where(tiny[0], np.nan, t)


def init_params(ngl, seed=0):
    """He-uniform weights, zero biases (padding columns of W1 zero)."""
    rng = np.random.default_rng(seed)
    L = layout(ngl)
    P = np.zeros(L["total"], dtype=np.float32)
    W1 = np.zeros((H, L["kp"]), dtype=np.float32)
    a1 = np.sqrt(6.0 / nin(ngl))
    W1[:, :nin(ngl)] = rng.uniform(-a1, a1, size=(H, nin(ngl)))
    a2 = np.sqrt(6.0 / H)
    P[L["w1"]:L["b1"]] = W1.ravel()
    P[L["w2"]:L["b2"]] = rng.uniform(-a2, a2, size=H * H)
    P[L["w3"]:L["b3"]] = rng.uniform(-np.sqrt(3.0 / H), np.sqrt(3.0 / H), size=H)
    return P


def forward(X, P, ngl, quantised=True):
    """Network output and the intermediates the backward pass needs."""
    W1, b1, W2, b2, w3, b3 = unpack(np.asarray(P, dtype=np.float32 if quantised else np.float64), ngl)
    q = bf16 if quantised else (lambda a: np.asarray(a, dtype=np.float64))
    X64 = np.asarray(X, dtype=np.float64)
    W1q, W2q = q(W1).astype(np.float64), q(W2).astype(np.float64)
    Z1 = X64 @ W1q.T + b1
    A1 = np.maximum(Z1, 0.0)
    A1q = bf16(A1.astype(np.float32)).astype(np.float64) if quantised else A1
    Z2 = A1q @ W2q.T + b2
    A2 = np.maximum(Z2, 0.0)
    y = A2 @ w3.astype(np.float64) + float(b3)
    return y, dict(X=X64, W2=W2q, Z1=Z1, A1=A1q, Z2=Z2, A2=A2, w3=w3.astype(np.float64))


def loss_and_grad(X, t, P, ngl, quantised=True):
    """(1/M) sum (y - t)^2 and its gradient (the roundings treated as identity)."""
    L = layout(ngl)
    y, c = forward(X, P, ngl, quantised)
    M = len(y)
    e = y - np.asarray(t, dtype=np.float64)
    dy = 2.0 * e / M
    G = np.zeros(L["total"], dtype=np.float64)
    G[L["b3"]] = dy.sum()
    G[L["w3"]:L["b3"]] = c["A2"].T @ dy
    dZ2 = np.outer(dy, c["w3"]) * (c["Z2"] > 0)
    G[L["b2"]:L["w3"]] = dZ2.sum(0)
    G[L["w2"]:L["b2"]] = (dZ2.T @ c["A1"]).ravel()
    dZ1 = (dZ2 @ c["W2"]) * (c["A1"] > 0)
    G[L["b1"]:L["w2"]] = dZ1.sum(0)
    gW1 = dZ1.T @ c["X"]
    gW1[:, nin(ngl):] = 0.0
    G[L["w1"]:L["b1"]] = gW1.ravel()
    return float((e * e).mean()), G


def adam(P, G, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, ngl=None):
    """One Adam step (Kingma & Ba 2015) in float32; padding slots untouched."""
    L = layout(ngl)
    idx = np.arange(L["total"])
    live = ~(((idx < L["b1"]) & ((idx % L["kp"]) >= nin(ngl))) | (idx > L["b3"]))
    P, m, v = P.copy(), m.copy(), v.copy()
    g = G.astype(np.float32)
    m[live] = b1 * m[live] + (1 - b1) * g[live]
    v[live] = b2 * v[live] + (1 - b2) * g[live] * g[live]
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    P[live] = P[live] - lr * (m[live] / c1) / (np.sqrt(v[live] / c2) + eps)
    return P, m, v
