"""The oracle against the reference program, live, on the problems the GPU
parity tests compare the engine with the oracle on (CPU).

tests/test_gpu_parity.py, test_gpu_av_pp.py and test_gpu_partial_dry.py
hold the engine to the oracle on rotated curved meshes (every
face-orientation pairing), NumFlux 3, SSP-RK3, the artificial-viscosity
path, and the partial-dry treatment with artificial viscosity.  Here the reference program
(oracle/_ref/esdg_ref) runs the same problems -- the mesh written as ISM-V2
by the engine's writer and read by the reference's reader, state and
bathymetry injected -- and the oracle must end in its state bit for bit, so
that engine == oracle == reference holds on those problems too.  Needs the
reference tree (the kernels of these parameter sets are built from it).
"""
import os
import shutil

import numpy as np
import pytest

from esdgsem_mpiocca_b200 import host, problems
from oracle import run_ref
from oracle.oracle import OracleProblem

pytestmark = pytest.mark.skipif(not run_ref.available(), reason="needs the reference tree")


def _ssp(pr):
    pr.params.rkOrder, pr.params.rkSSP = 3, 1
    pr.rkA, pr.rkB, pr.rkC = host.rk_coefficients(3, 1)
    return pr


def _island_av():
    """The partial-dry island of tests/golden/island_pd_N3.npz with the
    artificial viscosity on top (tests/test_gpu_partial_dry.py)."""
    import dataclasses
    from tests.golden import fixtures
    prob = fixtures.load("island_pd_N3")[0]
    p = dataclasses.replace(prob.params, ArtificialViscosity=1, epsilon_0=0.002, sigma_min=-6.0, sigma_max=-2.0,
                            DFL=0.1)
    fd = prob.basis.fd_mats
    prob = host.make_problem(p, prob.mesh, prob.b, prob.q0, prob.meta)
    prob.basis.fd_mats = fd
    return prob


CASES = {
    # (problem, mesh arguments as the problem builds its mesh, end time)
    "curved_rot_nf3_N3": (lambda: problems.curved_lake(N=3, nel=12, seed=3, ripple=0.02, NumFlux=3, rotate_seed=7),
                          dict(N=3, nel=12, rot=7), 0.01),
    "curved_rot_nf0_N4": (lambda: problems.curved_lake(N=4, nel=16, seed=1, ripple=0.05, rotate_seed=11),
                          dict(N=4, nel=16, rot=11), 0.01),
    "curved_rot_ssp_nf3_N3": (lambda: _ssp(problems.curved_lake(N=3, nel=12, seed=3, ripple=0.02, NumFlux=3,
                                                                rotate_seed=7)),
                              dict(N=3, nel=12, rot=7), 0.01),
    "dam_av_rot_N3": (lambda: problems.dam_break(N=3, nel=12, seed=2, rotate_seed=5), dict(N=3, nel=12, rot=5),
                      0.005),
    "dam_av_N4": (lambda: problems.dam_break(N=4, nel=12, seed=2), dict(N=4, nel=12, rot=0), 0.005),
    # Cartesian mesh of the reference's own generator: (xL, xR, yL, yR, NX, NY, periodic rows, columns)
    "island_pd_av_N3": (_island_av, dict(cart=(0.0, 1.0, 0.0, 1.0, 12, 12, 0, 0)), 0.004),
    # higher degrees on a rotated curved mesh
    "curved_rot_nf0_N5": (lambda: problems.curved_lake(N=5, nel=8, seed=5, ripple=0.05, rotate_seed=3),
                          dict(N=5, nel=8, rot=3), 0.01),
    "curved_rot_nf3_N6": (lambda: problems.curved_lake(N=6, nel=6, seed=6, ripple=0.05, NumFlux=3, rotate_seed=9),
                          dict(N=6, nel=6, rot=9), 0.01),
    "curved_rot_nf0_N7": (lambda: problems.curved_lake(N=7, nel=5, seed=7, ripple=0.05, rotate_seed=4),
                          dict(N=7, nel=5, rot=4), 0.01),
    # the lowest degrees: N = 1 (2x2 nodes) and N = 2 (tests/test_gpu_degrees.py)
    "curved_rot_nf0_N1": (lambda: problems.curved_lake(N=1, nel=12, seed=8, ripple=0.05, rotate_seed=6),
                          dict(N=1, nel=12, rot=6), 0.01),
    "curved_rot_nf3_N2": (lambda: problems.curved_lake(N=2, nel=10, seed=9, ripple=0.05, NumFlux=3, rotate_seed=2),
                          dict(N=2, nel=10, rot=2), 0.01),
    # the manufactured-solution test (Testcase 1) at N = 4 (tests/test_gpu_convergence.py)
    "conv_tc1_N4": (lambda: problems.conv_test(N=4, nel=6), dict(cart=(0.0, 2.0, 0.0, 2.0, 6, 6, 0, 0)), 0.02),
    # an ensemble member at its own scales: 2000 km square, 4000 m shelf, Okada uplift, viscosity on
    "tsunami_av_N3": (lambda: problems.tsunami_member(3, N=3, steps=0, sizes=(16,)),
                      dict(cart=(0.0, 2.0e6, 0.0, 2.0e6, 16, 16, 0, 0)), 300.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_program(name, tmp_path):
    make, m, T = CASES[name]
    pr = make()
    if "cart" in m:
        where = dict(cartesian=m["cart"])
    else:
        path = str(tmp_path / f"{name}.mesh")
        mesh = host.mesh_mapped(m["N"], 0.0, 1.0, 0.0, 1.0, m["nel"], m["nel"], amp=0.03, rotate_seed=m["rot"],
                                write_path=path)
        np.testing.assert_array_equal(mesh.x, pr.mesh.x)  # the problem's own mesh
        where = dict(mesh_file=path)
    p = pr.params
    p.T = T
    try:
        out = run_ref.run(f"live_{name}", p, inject={"q": pr.q0, "b": pr.b, "Bx": pr.Bx, "By": pr.By}, **where)
    finally:
        shutil.rmtree(os.path.join(run_ref.HERE, "_ref", "runs", f"live_{name}"), ignore_errors=True)
    ref = OracleProblem(pr).run(T=T, max_steps=0)
    assert ref["steps"] >= 3
    np.testing.assert_array_equal(ref["q"], out["q_final"])
