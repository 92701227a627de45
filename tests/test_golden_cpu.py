"""Pins the oracle and the host set-up to the reference itself (CPU).

The fixtures in tests/golden/ come from runs of the reference program
(tests/golden/make_golden.py).  Required here:
  * the oracle started from the reference's own copyDeviceVariables arrays
    ends in exactly the reference's final state (bit for bit: both are plain
    double arithmetic in the same order, no FMA contraction);
  * the engine's host set-up (basis, Cartesian generator, ISM-V2 reader of
    its own curved meshes, element sizes, packed tables) reproduces the
    reference's set-up arrays bit for bit.
"""
import os

import numpy as np
import pytest

from esdgsem_mpiocca_b200 import host
from oracle.oracle import OracleProblem
from tests.golden import fixtures

CASES = [n for n in fixtures.names() if not n.startswith("okada")]


def test_fixtures_present():
    assert len(CASES) >= 7


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_bitwise(name):
    prob, q_ref, _ = fixtures.load(name)
    out = OracleProblem(prob).run(T=prob.params.T, max_steps=0)
    assert out["steps"] > 0
    assert np.isfinite(q_ref).all()
    np.testing.assert_array_equal(out["q"], q_ref)


def test_oracle_reproduces_reference_analysis_outputs():
    """Arrival times and maximum elevation (okl/Analysis/*), updated after
    every step, equal the arrays the reference's DGtimeloop read back at its
    end, bit for bit; the ripple reached part of the lake and not all of it."""
    prob, q_ref, z = fixtures.load("walls_analysis_N3")
    out = OracleProblem(prob).run(T=prob.params.T, max_steps=0)
    np.testing.assert_array_equal(out["q"], q_ref)
    np.testing.assert_array_equal(out["ArrivalTimings"], z["ArrivalTimings"])
    np.testing.assert_array_equal(out["MaximumElevation"], z["MaximumElevation"])
    at = z["ArrivalTimings"]
    assert 0 < (at == 1000.0).sum() < at.size
    assert len(np.unique(at[at < 1000.0])) > 10  # arrivals spread over many steps
    assert z["MaximumElevation"].max() > 0.005


@pytest.mark.parametrize("N", [2, 3, 4])
def test_basis_matches_reference(N):
    name = {2: "walls_ssp3_N2", 3: "periodic_nf0_N3", 4: "mapped_rot_N4"}[N]
    _, _, z = fixtures.load(name)
    b = host.Basis.build(N)
    for k, mine in (("D", b.D), ("Dstrong", b.Dstrong), ("Dhat", b.Dhat), ("VdmInv", b.VdmInv)):
        np.testing.assert_array_equal(mine, z[k], err_msg=k)


def test_partial_dry_matrices_match_reference():
    """esdg_basis_fd against the matrices the reference handed to
    copyPartialDryData (basis::FiniteDifferenceOperators)."""
    _, _, z = fixtures.load("island_pd_N3")
    Dc, Df, Db = host.Basis.build(3).fd()
    np.testing.assert_array_equal(Dc, z["DcFD"])
    np.testing.assert_array_equal(Df, z["DfFD"])
    np.testing.assert_array_equal(Db, z["DbFD"])


def test_partial_dry_changes_the_run():
    """The island case exercises the treatment: without it the oracle ends
    elsewhere than the reference."""
    prob, q_ref, _ = fixtures.load("island_pd_N3")
    prob.params.PartialDryTreatment = 0
    out = OracleProblem(prob).run(T=prob.params.T, max_steps=0)
    assert np.abs(out["q"] - q_ref).max() > 1e-3


def _compare_setup(mesh, basis, z, skip=()):
    es, _ = host.element_sizes(mesh, basis)
    pairs = [("nx", mesh.nx), ("ny", mesh.ny), ("scal", mesh.scal), ("x_xi", mesh.x_xi), ("x_eta", mesh.x_eta),
             ("y_xi", mesh.y_xi), ("y_eta", mesh.y_eta), ("Jinv", mesh.Jinv), ("x", mesh.x), ("y", mesh.y),
             ("EleSizes", es), ("EdgeData", mesh.EdgeData), ("EdgeReversed", mesh.EdgeReversed),
             ("ElemToEdge", mesh.ElemToEdge), ("MasterSlave", mesh.MasterSlave), ("Orientation", mesh.Orientation)]
    for k, mine in pairs:
        if k in skip:
            continue
        np.testing.assert_array_equal(mine, z[k].astype(mine.dtype), err_msg=k)


@pytest.mark.parametrize("name,args", [
    ("periodic_nf0_N3", (3, 0.0, 2.0, 0.0, 2.0, 16, 16, True, True)),
    ("walls_ssp3_N2", (2, -1.0, 1.0, 0.0, 1.0, 10, 8, False, False)),
])
def test_cartesian_setup_matches_reference(name, args):
    _, _, z = fixtures.load(name)
    mesh = host.mesh_cartesian(*args)
    _compare_setup(mesh, host.Basis.build(args[0]), z)


def test_curved_rotated_setup_matches_reference_reader():
    # the reference read the ISM-V2 file that this generator writes
    _, _, z = fixtures.load("mapped_rot_N4")
    mesh = host.mesh_mapped(4, 0.0, 1.0, 0.0, 1.0, 8, 8, amp=0.03, curve_order=5, rotate_seed=7)
    assert (mesh.EdgeReversed == 0).any()
    _compare_setup(mesh, host.Basis.build(4), z)


def test_ism2_roundtrip(tmp_path):
    p = tmp_path / "m.mesh"
    a = host.mesh_mapped(3, 0.0, 2.0, -1.0, 1.0, 5, 4, amp=0.05, curve_order=4, rotate_seed=3, write_path=p)
    b = host.mesh_read(3, p)
    for k in ("x", "y", "x_xi", "x_eta", "y_xi", "y_eta", "Jinv", "nx", "ny", "scal", "EdgeData", "ElemToEdge",
              "MasterSlave", "Orientation", "EdgeReversed"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)


def test_bottom_derivatives_match_reference_algorithm():
    # Bx/By recomputed on the reference's geometry equal the injected ones
    prob, _, z = fixtures.load("circle_lake_N3")
    Bx, By = host.bottom_derivatives(prob.mesh, prob.basis, z["b"])
    np.testing.assert_array_equal(Bx, z["Bx"])
    np.testing.assert_array_equal(By, z["By"])


@pytest.mark.skipif(not __import__("oracle.run_ref", fromlist=["available"]).available(),
                    reason="reference tree not present")
@pytest.mark.parametrize("fixture,mesh_file,N", [("circle_lake_N3", "CircleInCircle.mesh", 3),
                                                  ("curvedam_N3", "CurveDamN3.mesh", 3),
                                                  ("pxy4_lake_N4", "PeriodicXandY4.mesh", 4)])
def test_reader_matches_reference_on_shipped_curved_mesh(fixture, mesh_file, N):
    """Mesh::ReadMesh on the reference's own meshes (CircleInCircle.mesh:
    curved boundaries of order 6, 83 reversed faces; CurveDamN3.mesh: 1600
    elements, order 3; PeriodicXandY4.mesh: 16 elements, order 4) vs the
    engine's reader."""
    import os
    from oracle import run_ref
    _, _, z = fixtures.load(fixture)
    mesh = host.mesh_read(N, os.path.join(run_ref.REF, "meshFiles", mesh_file))
    _compare_setup(mesh, host.Basis.build(N), z)


def test_okada_matches_reference_routine():
    """Okada uplift restated in esdgsem_mpiocca_b200/okada.py vs the
    reference's src/okada.cpp run on its shipped fault file (fixture)."""
    from esdgsem_mpiocca_b200 import okada
    z = np.load(os.path.join(os.path.dirname(fixtures.__file__), "okada_fault1.npz"))
    # file order: lon, lat, depth, length, width, strike, slip(rake), dip, dislocation
    lon, lat, depth, length, width, strike, rake, dip, slip = z["fault"]
    f = okada.Fault(lon, lat, depth, length, width, strike, rake, dip, slip)
    mine = okada.uplift_mercator(z["x_km"], z["y_km"], f)
    ref = z["uplift_km"]
    assert (ref != 0).sum() > 1000
    np.testing.assert_array_equal(mine != 0, ref != 0)
    assert np.abs(mine - ref).max() <= 1e-12 * np.abs(ref).max()


def test_oracle_reproduces_reference_errors_on_testcase1():
    """Testcase 1: the reference prints its errors against the exact
    solution; the oracle's final state gives the same Linf errors."""
    import json
    import re
    from esdgsem_mpiocca_b200 import problems
    prob, q_ref, z = fixtures.load("conv_tc1_N3")
    out = OracleProblem(prob).run(T=prob.params.T, max_steps=0)
    tail = json.loads(bytes(z["meta"]).decode())["reference_stdout_tail"]
    printed = [float(v) for v in re.findall(r"LinfError\[\d\] is: ([0-9.eE+-]+)", tail)]
    assert len(printed) == 3
    d = np.abs(out["q"] - problems.conv_exact(prob, out["t"])).reshape(prob.K, 3, -1)
    for v in range(3):
        assert abs(d[:, v].max() - printed[v]) <= 1e-9 * printed[v], (v, d[:, v].max(), printed[v])


def test_oracle_converges_at_order_on_testcase1():
    """The manufactured solution's L2 error in h falls at order N+1."""
    from esdgsem_mpiocca_b200 import problems
    errs = []
    for nel in (4, 8):
        pr = problems.conv_test(N=3, nel=nel, T=0.1, CFL=0.2)
        out = OracleProblem(pr).run(T=0.1, max_steps=0)
        d = (out["q"] - problems.conv_exact(pr, out["t"])).reshape(pr.K, 3, -1)
        w = np.outer(pr.basis.wGL, pr.basis.wGL).reshape(-1)
        J = 1.0 / pr.mesh.Jinv.reshape(pr.K, -1)
        errs.append(float(np.sqrt(((d[:, 0] ** 2) * w * J).sum())))
    assert np.log2(errs[0] / errs[1]) >= 3.5, errs
