"""The oracle against the reference program, live, on the problems the GPU
parity tests compare the engine with the oracle on (CPU).

tests/test_gpu_parity.py and test_gpu_av_pp.py hold the engine to the
oracle on rotated curved meshes (every face-orientation pairing), NumFlux 3,
SSP-RK3 and the artificial-viscosity path.  Here the reference program
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
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_program(name, tmp_path):
    make, m, T = CASES[name]
    pr = make()
    path = str(tmp_path / f"{name}.mesh")
    mesh = host.mesh_mapped(m["N"], 0.0, 1.0, 0.0, 1.0, m["nel"], m["nel"], amp=0.03, rotate_seed=m["rot"],
                            write_path=path)
    np.testing.assert_array_equal(mesh.x, pr.mesh.x)  # the problem's own mesh
    p = pr.params
    p.T = T
    try:
        out = run_ref.run(f"live_{name}", p, mesh_file=path,
                          inject={"q": pr.q0, "b": pr.b, "Bx": pr.Bx, "By": pr.By})
    finally:
        shutil.rmtree(os.path.join(run_ref.HERE, "_ref", "runs", f"live_{name}"), ignore_errors=True)
    ref = OracleProblem(pr).run(T=T, max_steps=0)
    assert ref["steps"] >= 3
    np.testing.assert_array_equal(ref["q"], out["q_final"])
