"""Partial-dry treatment (PartialDryTreatment = 1) on the GPU against the
oracle (GPU).  The reference's own run of the island case is checked by
tests/test_gpu_golden.py; here: one right-hand side, artificial viscosity
on top of the treatment, every element-kernel variant, and the call order
the reference requires (copyPartialDryData before the first step).
"""
import dataclasses

import numpy as np
import pytest

from esdgsem_mpiocca_b200 import host
from esdgsem_mpiocca_b200.deviceclass import E_ARG, EsdgError, Solver
from oracle.oracle import OracleProblem
from tests.golden import fixtures

pytestmark = pytest.mark.gpu


def _island(**kw):
    prob, q_ref, _ = fixtures.load("island_pd_N3")
    if kw:
        p = dataclasses.replace(prob.params, **kw)
        fd = prob.basis.fd_mats
        prob = host.make_problem(p, prob.mesh, prob.b, prob.q0, prob.meta)
        prob.basis.fd_mats = fd
    return prob


def test_partial_dry_rhs_bitwise():
    prob = _island()
    s = Solver(prob)
    try:
        Qt = s.rhs()
    finally:
        s.close()
    ref = OracleProblem(prob).rhs(prob.q0)
    np.testing.assert_array_equal(Qt, ref)


def test_partial_dry_with_artificial_viscosity():
    prob = _island(ArtificialViscosity=1, epsilon_0=0.002, sigma_min=-6.0, sigma_max=-2.0, DFL=0.1)
    s = Solver(prob)
    try:
        s.run(T=1e9, max_steps=15)
        q = s.q()
    finally:
        s.close()
    ref = OracleProblem(prob).run(T=1e9, max_steps=15)["q"]
    K, n2 = prob.K, prob.ngl ** 2
    a, b = q.reshape(K, 3, n2), ref.reshape(K, 3, n2)
    for v in range(3):
        err = np.linalg.norm(a[:, v] - b[:, v]) / max(np.linalg.norm(b[:, v]), 1e-300)
        assert err <= 1e-12, (v, err)


def test_partial_dry_every_element_variant():
    prob = _island()
    out = {}
    for v in range(5):
        s = Solver(prob)
        try:
            try:
                s.dc.set_element_variant(v)
            except EsdgError:
                continue
            s.run(T=prob.params.T, max_steps=0)
            out[v] = s.q()
        finally:
            s.close()
    assert {0, 3, 4} <= set(out)
    for v, q in out.items():
        np.testing.assert_array_equal(q, out[0], err_msg=f"variant {v}")


def test_partial_dry_needs_its_matrices():
    prob = _island()
    p, m, bs = prob.params, prob.mesh, prob.basis
    from esdgsem_mpiocca_b200.deviceclass import DeviceClass
    dc = DeviceClass(0, -1)
    try:
        dc.initDeviceVariables(p.N, m.K, m.F, 0, p.rkSSP, p.NEpad, p.NEsurfpad, p.Nedgepad, p.NavgPad, p.ES,
                               p.Testcase, p.epsilon_0, p.sigma_max, p.sigma_min, p.PosPresTOL, bs.geomface,
                               p.g_const, p.PositivityPreserving, p.ArtificialViscosity, p.DiscBottom, 0.0, 1, 0, 0,
                               0, 0)
        zeros = np.zeros_like(prob.q0)
        dc.copyDeviceVariables(p.PositivityPreserving, m.K, bs.wGL, m.nx, m.ny, m.scal, m.y_xi, m.y_eta, m.x_xi,
                               m.x_eta, prob.b, prob.Bx, prob.By, bs.D, bs.Dstrong, bs.Dhat, m.Jinv, m.x, m.y,
                               prob.q0, prob.EleSizes, zeros, zeros, bs.VdmInv, m.MasterSlave, m.Orientation,
                               m.ElemToEdge, m.EdgeData, m.EdgeReversed)
        dc.buildDeviceKernels(99, 99, p.Testcase, p.FluxDifferencing, p.NumFlux, p.rkSSP, p.ArtificialViscosity,
                              p.PositivityPreserving, p.DiscBottom)
        with pytest.raises(EsdgError) as ei:
            dc.compute_rhs(prob.K, prob.ngl, False)
        assert ei.value.code == E_ARG
        dc.copyPartialDryData(*bs.fd_mats)
        Qt = dc.compute_rhs(prob.K, prob.ngl, False)
        assert np.isfinite(Qt).all()
    finally:
        dc.close()
