"""The C-ABI library (CPU, no GPU calls): it loads, exports every function
include/esdg_b200.h declares, and its host set-up entry points behave."""
import os
import re
import subprocess

import numpy as np
import pytest

import esdgsem_mpiocca_b200 as pkg
from esdgsem_mpiocca_b200 import host

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(esdg_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_every_declared_symbol():
    L = pkg.lib()
    names = declared("esdg_b200.h")
    assert len(names) >= 29
    out = subprocess.run(["nm", "-D", "--defined-only", pkg.library_path()], capture_output=True, text=True,
                         check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(L, n)


def test_device_entry_points_reject_null_handle():
    L = pkg.lib()
    assert L.esdg_copy_q_to_host(None, None) == -1
    assert L.esdg_dg_timeloop(None, 1, 1, 5, None, None, None, 1.0, 0.4, 0.1, 1.0, 0, 0, 0, 0, 0, 9.81, 0, 0, 0,
                              0, 0, None, None) == -1
    assert L.esdg_bytes_allocated(None) == -1


def test_rk_tables():
    A, B, C = host.rk_coefficients(4, 0)
    assert len(A) == 5 and A[0] == 0.0 and B[0] == 0.0
    # 2N-storage consistency: the stage times are B (Carpenter-Kennedy)
    np.testing.assert_allclose(B[-1], 2802321613138.0 / 2924317926251.0)
    A3, B3, C3 = host.rk_coefficients(3, 1)
    assert list(A3) == [1.0, 0.75, 1.0 / 3.0]


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_basis_properties(N):
    b = host.Basis.build(N)
    n = N + 1
    D0 = b.D0.reshape(n, n)
    # exact on polynomials of degree <= N
    for k in range(n):
        np.testing.assert_allclose(D0 @ b.xGL ** k, k * b.xGL ** max(k - 1, 0) if k else 0 * b.xGL, atol=1e-11)
    # summation-by-parts: M D + D^T M = diag(-1, 0, ..., 0, 1)
    M = np.diag(b.wGL)
    Q = M @ D0 + D0.T @ M
    E = np.zeros((n, n))
    E[0, 0], E[-1, -1] = -1.0, 1.0
    np.testing.assert_allclose(Q, E, atol=1e-12)
    assert abs(b.wGL.sum() - 2.0) < 1e-14 and abs(b.wG.sum() - 2.0) < 1e-14
    # modal transform maps nodal Legendre polynomials to unit vectors
    from numpy.polynomial import legendre
    V = b.VdmInv.reshape(n, n)
    for j in range(n):
        c = np.zeros(j + 1)
        c[j] = 1.0
        nodal = legendre.legval(b.xGL, c) * np.sqrt(j + 0.5)   # orthonormal Legendre mode j
        e = V @ nodal
        np.testing.assert_allclose(e, np.eye(n)[j], atol=1e-11)


def test_mapped_mesh_metric_identities_and_faces():
    N = 4
    m = host.mesh_mapped(N, 0.0, 1.0, 0.0, 1.0, 6, 5, amp=0.03, curve_order=6, rotate_seed=9)
    b = host.Basis.build(N)
    n = N + 1
    D0 = b.D0.reshape(n, n)
    for arr in ("x_xi", "x_eta", "y_xi", "y_eta"):
        assert np.isfinite(getattr(m, arr)).all()
    # discrete metric identities: d_xi(y_eta) - d_eta(y_xi) = 0 on every element
    ye = m.y_eta.reshape(m.K, n, n)
    yx = m.y_xi.reshape(m.K, n, n)
    err = np.einsum("ik,ejk->eji", D0, ye) - np.einsum("jk,eki->eji", D0, yx)
    assert np.abs(err).max() < 1e-12
    # unit normals, positive Jacobians
    assert np.allclose(m.nx ** 2 + m.ny ** 2, 1.0)
    assert (m.Jinv > 0).all()
    # every element side has a face and interior faces have two elements
    ED = m.EdgeData.reshape(m.F, 8)
    nb = (ED[:, 1] == -1).sum()
    assert nb == 2 * (6 + 5)
    assert (m.ElemToEdge >= 1).all() and (m.ElemToEdge <= m.F).all()


def test_cartesian_periodic_counts():
    m = host.mesh_cartesian(3, 0.0, 2.0, 0.0, 2.0, 16, 16, True, True)
    assert m.K == 256 and m.F == 512
    assert (m.EdgeData.reshape(-1, 8)[:, 6] == 0).all()   # no wall faces
    m2 = host.mesh_cartesian(3, 0.0, 2.0, 0.0, 1.0, 4, 3)
    assert m2.F == 5 * 3 + 4 * 4


def test_mesh_read_errors_are_reported(tmp_path):
    bad = tmp_path / "bad.mesh"
    bad.write_text("ISM-V2\n3 2\n")
    with pytest.raises(RuntimeError):
        host.mesh_read(3, bad)
    with pytest.raises(RuntimeError):
        host.mesh_read(3, tmp_path / "missing.mesh")
