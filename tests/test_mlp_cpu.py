"""The learned indicator's CPU oracle (oracle/mlp_oracle.py), checked on its
own: its analytic gradient against central finite differences, its feature
map's invariances, its sensor value against the C restatement of the
reference's shock-capturing kernel, and the library's MLP entry points
being exported (no GPU needed)."""
import ctypes

import numpy as np
import pytest

from oracle import mlp_oracle as mo


@pytest.mark.parametrize("ngl", [4, 5])
def test_gradient_matches_finite_differences(ngl):
    rng = np.random.default_rng(1)
    M = 40
    X = rng.normal(size=(M, mo.kp(ngl)))
    X[:, mo.nin(ngl):] = 0.0
    t = rng.normal(size=M)
    P = mo.init_params(ngl, seed=3).astype(np.float64)
    L = mo.layout(ngl)
    P[L["b1"]:L["w2"]] = rng.normal(scale=0.1, size=mo.H)
    P[L["b2"]:L["w3"]] = rng.normal(scale=0.1, size=mo.H)
    _, G = mo.loss_and_grad(X, t, P, ngl, quantised=False)
    live = [i for i in range(L["b3"] + 1) if not (i < L["b1"] and i % L["kp"] >= mo.nin(ngl))]
    idx = rng.choice(live, size=60, replace=False).tolist() + [L["b3"], L["w3"], L["b2"], L["b1"]]
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (mo.loss_and_grad(X, t, Pp, ngl, False)[0] - mo.loss_and_grad(X, t, Pm, ngl, False)[0]) / (2 * h)
        assert abs(fd - G[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, G[i])


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38, 1e-40], dtype=np.float32)
    r = mo.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2 ** -7) and r[3] == -2.5
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)


def test_features_are_scale_and_offset_free_but_s_is_not():
    ngl = 5
    rng = np.random.default_rng(0)
    K, n2 = 16, 25
    q = rng.normal(size=(K, 3, n2))
    b = rng.normal(size=(K, n2))
    X1, s1 = mo.features(q, b, ngl)
    q2 = q.copy()
    q2[:, 1:, :] *= 7.0
    X2, _ = mo.features(q2, b, ngl)
    np.testing.assert_array_equal(X1[:, n2:3 * n2], X2[:, n2:3 * n2])
    q3 = q.copy()
    q3[:, 0, :] += 100.0       # eta shifted: shape features unchanged, s_eta drops
    X3, s3 = mo.features(q3, b, ngl)
    np.testing.assert_allclose(X1[:, :n2], X3[:, :n2], atol=2e-2)
    assert (s3 < s1).all()


def test_sigma_matches_c_restatement_of_the_sensor():
    """sigma from mlp_oracle gives the same viscosity as the C oracle's
    shock-capturing kernel (ramp of okl/ShockCapturing/ShockCapturing.okl)."""
    from esdgsem_mpiocca_b200 import host
    from oracle.oracle import _p, lib
    N = 4
    ngl = N + 1
    B = host.Basis.build(N)
    rng = np.random.default_rng(5)
    K, n2 = 200, ngl * ngl
    q = np.zeros((K, 3, n2))
    q[:, 0, :] = 1.0 + rng.normal(size=(K, n2)) * np.logspace(-6, -0.5, K)[:, None]
    b = np.zeros((K, n2))
    eps0, smin, smax = 0.7, -6.0, -2.0
    visc = np.zeros(K)
    lib().oracle_shock_capturing(N, K, eps0, smin, smax, _p(np.ascontiguousarray(q.ravel())), _p(b.ravel()),
                                 _p(np.ascontiguousarray(B.VdmInv)), _p(visc))
    sg = mo.sensor_sigma(q[:, 0, :] + b, B.VdmInv.reshape(ngl, ngl))
    ramp = np.where(sg <= smin, 0.0,
                    np.where(sg <= smax, 0.5 * eps0 * (1 + np.sin(np.pi * (sg - 0.5 * (smax + smin)) / (smax - smin))),
                             eps0))
    assert ((visc > 0) & (visc < eps0)).sum() > 20
    np.testing.assert_allclose(ramp, visc, rtol=1e-9, atol=1e-12)


def test_library_exports_mlp_entries():
    import esdgsem_mpiocca_b200 as pkg
    L = pkg.lib()
    out = (ctypes.c_int * 8)()
    assert L.esdg_mlp_layout(5, out) == 0
    lay = mo.layout(5)
    assert list(out) == [lay[k] for k in ("kp", "w1", "b1", "w2", "b2", "w3", "b3", "total")]
    assert L.esdg_mlp_layout(9, out) != 0
