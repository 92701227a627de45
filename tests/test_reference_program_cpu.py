"""The reference program as the benchmark's CPU baseline and reference arm (CPU).

bench.py times the reference program itself (oracle/_ref/esdg_ref) on the
host cores, with inputs made by NumPy alone (oracle/ref_inputs.py) and the
bathymetry and initial state set by the case hook at the reference's own
nodes (oracle/ref_shim/bench_case.cpp).  Where the benchmark runs, the
reference's .okl tree is absent; the OCCA stand-in then loads the kernels
built for the benchmark's parameters by their index key.  Required here:
* the NumPy mesh writer writes the engine writer's bytes;
* run that way on a small mesh, the program takes the requested number of
  steps (counted by the stand-in) and ends in the oracle's state, within the
  last-place differences of NumPy's and the C library's exp in the bumps.
"""
import filecmp
import os

import numpy as np
import pytest

import bench
from esdgsem_mpiocca_b200 import host, problems
from oracle import ref_inputs, run_ref
from oracle.oracle import OracleProblem


@pytest.mark.parametrize("nel", [3, 8, 16])
def test_numpy_mesh_writer_matches_engine_writer(tmp_path, nel):
    a, b = str(tmp_path / "numpy.mesh"), str(tmp_path / "engine.mesh")
    K, F = ref_inputs.write_mapped_mesh(a, nel)
    host.mesh_mapped(bench.N_POLY, 0.0, 1.0, 0.0, 1.0, nel, nel, amp=0.03, write_path=b)
    assert (K, F) == (nel * nel, 2 * nel * (nel + 1))
    assert filecmp.cmp(a, b, shallow=False)


def test_case_state_matches_engine_problem():
    pr = problems.curved_lake(N=bench.N_POLY, nel=8, steps=0)
    b, h = ref_inputs.case_state(pr.mesh.x, pr.mesh.y, 0)
    np.testing.assert_array_equal(b, pr.b)
    np.testing.assert_array_equal(h, pr.q0.reshape(pr.K, 3, -1)[:, 0].reshape(-1))


def test_lake_params_take_the_requested_steps():
    """T of lake_params gives the oracle, on the engine's problem, exactly
    the requested number of steps."""
    pr = problems.curved_lake(N=bench.N_POLY, nel=16, steps=0)
    for n in (3, 7):
        p = ref_inputs.lake_params(16, bench.N_POLY, n)
        assert OracleProblem(pr).run(T=p.T, max_steps=0)["steps"] == n


@pytest.mark.skipif(not os.path.exists(run_ref.EXE), reason="reference program not built")
def test_reference_program_runs_from_prebuilt_kernels(tmp_path, monkeypatch):
    nel = 8
    pr = problems.curved_lake(N=bench.N_POLY, nel=nel, steps=0)
    mesh, case = str(tmp_path / "lake8.mesh"), str(tmp_path / "case.txt")
    ref_inputs.write_mapped_mesh(mesh, nel)
    ref_inputs.write_case(case, 0)
    p = ref_inputs.lake_params(nel, bench.N_POLY, 5)
    if run_ref.available():  # build the benchmark's kernels here, as build() does
        run_ref.warm_kernels(p, mesh)
    monkeypatch.setattr(run_ref, "REF", str(tmp_path / "no-reference-tree"))
    assert not run_ref.available()
    try:
        sec, out, q = run_ref.run_timed(p, mesh, None, threads=2, want_q=True,
                                        extra_env={"ESDG_REF_CASE": case, "ESDG_REF_COUNT": "1"})
    except RuntimeError as e:
        if "no prebuilt kernel" in str(e):
            pytest.skip("the benchmark's reference kernels were not built (needs the reference tree once)")
        raise
    assert sec > 0
    assert run_ref.kernel_calls(out)["FindLambdaMax"] == 5
    ref = OracleProblem(pr).run(T=p.T, max_steps=0)
    assert ref["steps"] == 5
    qa, qb = q.reshape(pr.K, 3, -1), ref["q"].reshape(pr.K, 3, -1)
    scale = np.abs(qb[:, 0]).max()
    for v in range(3):
        assert np.abs(qa[:, v] - qb[:, v]).max() <= 1e-13 * scale, v


def test_reference_arm_loads_nothing_of_the_engine():
    """The reference arm's process imports no module of the engine and maps
    no shared library of this repository while it prepares the reference
    program's inputs."""
    import subprocess
    import sys
    code = (
        "import os, sys, tempfile; sys.path.insert(0, os.getcwd()); import bench\n"
        "from oracle import ref_inputs, run_ref\n"
        "d = tempfile.mkdtemp(); ref_inputs.write_mapped_mesh(d + '/m.mesh', 4); ref_inputs.write_case(d + '/c', 0)\n"
        "p = ref_inputs.lake_params(4, bench.N_POLY, 3); c = bench.workload_config()\n"
        "assert not any(m.startswith('esdgsem_mpiocca_b200') for m in sys.modules), sorted(sys.modules)\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libesdg_b200' not in maps and 'libesdg_oracle' not in maps\n"
        "print('clean')\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "clean" in out.stdout
