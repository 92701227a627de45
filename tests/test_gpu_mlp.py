"""The learned indicator's CUDA kernels against the CPU oracle
(oracle/mlp_oracle.py): feature rows and sensor targets, the BF16
tensor-core forward pass, the backward pass (gradient of the mean squared
error), the Adam step, determinism of the gradient reduction, and that a
short training run on sensor-labelled solver states learns."""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.indicator import DeviceMLP, IndicatorNet
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _states(N, seed=0, K=None):
    """Element states of a dam break, perturbed so that sigma spans the
    sensor's range: (q [K][3][n2], b [K][n2], VdmInv)."""
    prob = problems.dam_break(N=N, nel=32, seed=seed)
    ngl = N + 1
    n2 = ngl * ngl
    rng = np.random.default_rng(seed)
    q = prob.q0.reshape(prob.K, 3, n2).copy()
    amp = np.logspace(-7, -1, prob.K)[rng.permutation(prob.K)]
    q[:, 0, :] += amp[:, None] * rng.normal(size=(prob.K, n2))
    q[:, 1, :] += 0.1 * rng.normal(size=(prob.K, 1)) + amp[:, None] * rng.normal(size=(prob.K, n2))
    q[:, 2, :] += amp[:, None] * rng.normal(size=(prob.K, n2))
    b = np.zeros((prob.K, n2))
    b[: prob.K // 3] = 0.3 * rng.normal(size=(prob.K // 3, 1))    # offset bathymetry in a third
    q[: prob.K // 3, 0, :] -= b[: prob.K // 3]
    b[5] = 0.0
    q[5, 0, :] = 1e-4                                            # below the energy threshold
    return q, b, prob.basis.VdmInv


def _dev(*arrs):
    import torch
    return [torch.tensor(np.ascontiguousarray(a), device="cuda") for a in arrs]


def _bf16_to_f32(X):
    import torch
    return X.float().cpu().numpy()


@pytest.mark.parametrize("N", [3, 4])
def test_features_and_targets_match_oracle(N):
    ngl = N + 1
    q, b, V = _states(N)
    qd, bd, Vd = _dev(q.ravel(), b.ravel(), V.ravel())
    mlp = DeviceMLP(IndicatorNet.fresh(ngl), 0)
    X, t, s = mlp.features(qd.data_ptr(), bd.data_ptr(), Vd.data_ptr(), q.shape[0])
    Xo, so = mo.features(q, b, ngl)
    to = mo.target(q, b, V.reshape(ngl, ngl), ngl)
    Xg = _bf16_to_f32(X)
    # identical up to one BF16 rounding step (statistics summed in another order)
    ulp = np.abs(Xo) * 2.0 ** -7 + 1e-30
    bad = np.argwhere(np.abs(Xg - Xo) > ulp)
    assert len(bad) == 0, [(int(i), int(j), float(Xg[i, j]), float(Xo[i, j])) for i, j in bad[:10]]
    assert (Xg == Xo).mean() > 0.99
    np.testing.assert_allclose(s.cpu().numpy(), so, rtol=0, atol=1e-5)
    tg = t.cpu().numpy()
    np.testing.assert_array_equal(np.isnan(tg), np.isnan(to))
    assert np.isnan(tg[5])
    ok = ~np.isnan(to)
    np.testing.assert_allclose(tg[ok], to[ok], rtol=0, atol=1e-4)
    sig = to[ok] + so[ok]
    assert sig.min() < -8 and sig.max() > -2   # the cases span the sensor's range


def _data(N, seed=0):
    ngl = N + 1
    q, b, V = _states(N, seed)
    Xo, so = mo.features(q, b, ngl)
    to = mo.target(q, b, V.reshape(ngl, ngl), ngl)
    ok = ~np.isnan(to)
    return Xo[ok], to[ok].astype(np.float32)


def _to_bf16(X):
    import torch
    return torch.tensor(X, device="cuda").to(torch.bfloat16)


@pytest.mark.parametrize("N", [3, 4])
def test_forward_matches_oracle(N):
    import torch
    ngl = N + 1
    X, _ = _data(N)
    net = IndicatorNet.fresh(ngl, seed=4)
    L = mo.layout(ngl)
    rng = np.random.default_rng(2)
    net.P[L["b1"]:L["w2"]] = rng.normal(scale=0.2, size=mo.H)
    net.P[L["b2"]:L["w3"]] = rng.normal(scale=0.2, size=mo.H)
    net.P[L["b3"]] = 0.3
    mlp = DeviceMLP(net, 0)
    y = mlp.forward(_to_bf16(X)).cpu().numpy()
    yo, _ = mo.forward(X, net.P, ngl)
    scale = np.abs(yo).max()
    assert scale > 0.1
    # FP32 accumulation order differs from the oracle's, so a hidden
    # activation can round to the neighbouring BF16 value now and then
    d = np.abs(y - yo)
    assert (d <= 1e-4 * scale).mean() >= 0.99, d.max()
    assert d.max() <= 2e-2 * scale, d.max()
    # rows not a multiple of 16 and a single row
    y7 = mlp.forward(_to_bf16(X[:7])).cpu().numpy()
    np.testing.assert_array_equal(y7, y[:7])
    torch.cuda.synchronize()


@pytest.mark.parametrize("N", [3, 4])
def test_backward_matches_oracle_and_is_deterministic(N):
    ngl = N + 1
    X, t = _data(N)
    net = IndicatorNet.fresh(ngl, seed=7)
    L = mo.layout(ngl)
    net.P[L["b1"]:L["w2"]] = 0.1
    net.P[L["b2"]:L["w3"]] = 0.1
    mlp = DeviceMLP(net, 0, blocks=16)
    Xd = _to_bf16(X)
    (td,) = _dev(t)
    G1, sse1 = mlp.gradient(Xd, td)
    G2, sse2 = mlp.gradient(Xd, td)
    G1 = G1.cpu().numpy()
    np.testing.assert_array_equal(G1, G2.cpu().numpy())
    loss_o, Go = mo.loss_and_grad(X, t, net.P, ngl)
    assert abs(float(sse1) / len(t) - loss_o) <= 1e-4 * loss_o
    live = np.r_[0:L["b3"] + 1]
    err = np.linalg.norm(G1[live] - Go[live]) / np.linalg.norm(Go[live])
    assert err < 2e-2, err
    for name, a, b_ in (("w1", "w1", "b1"), ("b1", "b1", "w2"), ("w2", "w2", "b2"), ("b2", "b2", "w3"),
                        ("w3", "w3", "b3")):
        g, o = G1[L[a]:L[b_]], Go[L[a]:L[b_]]
        assert np.linalg.norm(g - o) <= 3e-2 * np.linalg.norm(o) + 1e-9, name
    assert abs(G1[L["b3"]] - Go[L["b3"]]) <= 1e-3 * abs(Go[L["b3"]]) + 1e-7


def test_adam_step_matches_oracle():
    import torch
    ngl = 5
    X, t = _data(4)
    net = IndicatorNet.fresh(ngl, seed=1)
    mlp = DeviceMLP(net, 0, blocks=8)
    P0 = net.P.copy()
    m0 = np.zeros_like(P0)
    v0 = np.zeros_like(P0)
    (td,) = _dev(t)
    mlp.train_step(_to_bf16(X), td, 1e-3)
    G = mlp.G.cpu().numpy()
    Po, mo_, vo = mo.adam(P0, G, m0, v0, 1, 1e-3, ngl=ngl)
    np.testing.assert_allclose(mlp.P.cpu().numpy(), Po, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(mlp.m.cpu().numpy(), mo_, rtol=1e-6, atol=1e-12)
    L = mo.layout(ngl)
    pad = [i for i in range(L["b1"]) if i % L["kp"] >= mo.nin(ngl)]
    assert (mlp.P.cpu().numpy()[pad] == 0).all()
    assert (mlp.Pb.float().cpu().numpy() == mo.bf16(mlp.P.cpu().numpy())).all()
    torch.cuda.synchronize()


def test_short_training_learns_the_sensor():
    import torch
    N, ngl = 4, 5
    Xa, ta = [], []
    for seed in range(3):
        X, t = _data(N, seed)
        Xa.append(X)
        ta.append(t)
    X = np.concatenate(Xa)
    t = np.concatenate(ta)
    nval = len(t) // 5
    Xd, (td,) = _to_bf16(X), _dev(t)
    mlp = DeviceMLP(IndicatorNet.fresh(ngl, seed=0), 0, blocks=16)
    yv0 = mlp.forward(Xd[:nval])
    mse0 = float(((yv0 - td[:nval]) ** 2).mean())
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    M = len(t) - nval
    for it in range(600):
        idx = nval + torch.randint(0, M, (1024,), generator=g, device="cuda")
        mlp.train_step(Xd[idx].contiguous(), td[idx].contiguous(), 3e-3)
    yv = mlp.forward(Xd[:nval])
    mse = float(((yv - td[:nval]) ** 2).mean())
    assert mse < 0.3 * mse0, (mse0, mse)
