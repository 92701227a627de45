"""The reference program as the benchmark's CPU baseline (CPU).

bench.py times the reference program itself (oracle/_ref/esdg_ref) on the
host cores.  Where the benchmark runs, the reference's .okl tree is absent;
the OCCA stand-in then loads the kernels built for the benchmark's
parameters by their index key.  Required here: run that way, on the
benchmark's parameters over a small curved mesh written by the engine's
writer, the program takes the requested number of steps (its end time set
as bench.py sets it) and ends in the oracle's state bit for bit.
"""
import os

import numpy as np
import pytest

import bench
from esdgsem_mpiocca_b200 import host, problems
from oracle import run_ref
from oracle.oracle import OracleProblem

pytestmark = pytest.mark.skipif(not os.path.exists(run_ref.EXE), reason="reference program not built")


def test_reference_program_runs_from_prebuilt_kernels(tmp_path, monkeypatch):
    pr = problems.curved_lake(N=bench.N_POLY, nel=8, steps=0)
    path = str(tmp_path / "lake8.mesh")
    host.mesh_mapped(bench.N_POLY, 0.0, 1.0, 0.0, 1.0, 8, 8, amp=0.03, write_path=path)
    p = bench.reference_params(pr, 5)
    if run_ref.available():  # build the benchmark's kernels here, as build() does
        run_ref.warm_kernels(p, path)
    monkeypatch.setattr(run_ref, "REF", str(tmp_path / "no-reference-tree"))
    assert not run_ref.available()
    try:
        sec, out, q = run_ref.run_timed(p, path, {"q": pr.q0, "b": pr.b, "Bx": pr.Bx, "By": pr.By}, threads=2,
                                        want_q=True)
    except RuntimeError as e:
        if "no prebuilt kernel" in str(e):
            pytest.skip("the benchmark's reference kernels were not built (needs the reference tree once)")
        raise
    assert sec > 0
    ref = OracleProblem(pr).run(T=p.T, max_steps=0)
    assert ref["steps"] == 5
    np.testing.assert_array_equal(q, ref["q"])
