"""The reference's convergence test (Testcase 1: manufactured solution,
exact Dirichlet boundary states, source term) on the GPU.

* one right-hand side against the oracle (CUDA's and glibc's sin/cos may
  differ in the last place, so the bound is 1e-13 of the largest term);
* the engine's error against the exact solution falls at the scheme's order
  under refinement (about N+1: at least N+0.5 between successive meshes);
* the reference's own Testcase 1 run is checked in tests/test_gpu_golden.py
  (relative L2 <= 1e-12).
"""
import numpy as np
import pytest

from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.deviceclass import E_UNSUPPORTED, EsdgError, Solver
from oracle.oracle import OracleProblem

pytestmark = pytest.mark.gpu


def test_conv_rhs_matches_oracle():
    pr = problems.conv_test(N=4, nel=6)
    s = Solver(pr)
    try:
        Qg = s.rhs()
    finally:
        s.close()
    Qo = OracleProblem(pr).rhs(pr.q0)
    scale = np.abs(Qo).max() + 9.81 * 10 * 10
    assert np.abs(Qg - Qo).max() <= 1e-13 * scale


def _error(N, nel, T=0.1):
    pr = problems.conv_test(N=N, nel=nel, T=T, CFL=0.2)
    s = Solver(pr)
    try:
        t, _ = s.run(T=T, max_steps=0)
        q = s.q()
    finally:
        s.close()
    assert t == pytest.approx(T, abs=1e-14)
    ex = problems.conv_exact(pr, t)
    K, n2 = pr.K, (N + 1) ** 2
    w = np.outer(pr.basis.wGL, pr.basis.wGL).reshape(-1)
    d = (q - ex).reshape(K, 3, n2)
    J = 1.0 / pr.mesh.Jinv.reshape(K, n2)
    return float(np.sqrt(((d[:, 0] ** 2) * w * J).sum()))


@pytest.mark.parametrize("N,nels", [(3, (4, 8, 16)), (4, (4, 8))])
def test_manufactured_solution_converges_at_order(N, nels):
    errs = [_error(N, n) for n in nels]
    rates = [np.log2(errs[k] / errs[k + 1]) for k in range(len(errs) - 1)]
    assert errs[-1] < 1e-5, errs
    assert min(rates) >= N + 0.5, (errs, rates)


def test_conv_with_artificial_viscosity_is_rejected():
    pr = problems.conv_test(N=3, nel=4)
    pr.params.ArtificialViscosity = 1
    with pytest.raises(EsdgError) as ei:
        Solver(pr)
    assert ei.value.code == E_UNSUPPORTED
