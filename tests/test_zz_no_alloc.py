"""The allocation-free right-hand side (esdg_compute_rhs_noalloc) against the
ordinary one (esdg_compute_rhs) on the GPU.

Callers that cannot allocate device memory -- hosts that own all device
memory through their own pool, serving loops that must not synchronise the
device with cudaMalloc/cudaFree -- use the no-alloc entry point with buffers
they already hold.  Here torch provides those buffers; the entry point
itself allocates nothing.  Both entry points run the same kernels on the
same inputs, so the results must be identical (the tolerance of the other
engine tests, 1e-13 of the term scale, is met with equality), on two calls
in a row.  A corrupted connectivity entry is replaced by a safe one and
reported as ESDG_E_ARG.  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import esdgsem_mpiocca_b200 as pkg
from esdgsem_mpiocca_b200 import problems
from esdgsem_mpiocca_b200.deviceclass import Solver

pytestmark = pytest.mark.gpu


def _device_inputs(pr, torch):
    m, bs = pr.mesh, pr.basis
    dev = torch.device("cuda", 0)
    f64 = [pr.q0, m.Jinv, m.y_xi, m.y_eta, m.x_xi, m.x_eta, pr.Bx, pr.By, pr.b, bs.D, m.nx, m.ny, m.scal]
    i32 = [m.EdgeData, m.ElemToEdge, m.MasterSlave, m.Orientation]
    t64 = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev) for a in f64]
    t32 = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).to(dev) for a in i32]
    return t64, t32


def _noalloc_call(pr, t64, t32, torch):
    L = pkg.lib()
    p = pr.params
    out = torch.full((pr.q0.size,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.esdg_compute_rhs_noalloc(p.N, pr.K, pr.F, p.NumFlux, p.ES, p.g_const, p.PosPresTOL,
                                    *[ctypes.c_void_p(t.data_ptr()) for t in t64],
                                    *[ctypes.c_void_p(t.data_ptr()) for t in t32],
                                    ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    return rc, out.cpu().numpy()


def _noalloc_rhs(pr, t64, t32, torch):
    rc, out = _noalloc_call(pr, t64, t32, torch)
    assert rc == 0, pkg.lib().esdg_last_error(None).decode()
    return out


@pytest.mark.parametrize("case", ["periodic", "curved", "periodic_N2"])
def test_noalloc_rhs_matches_compute_rhs_twice(case):
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    if case == "periodic":
        pr = problems.periodic_bump(NumFlux=2, steps=0)
    elif case == "periodic_N2":
        pr = problems.periodic_bump(N=2, nel=12, NumFlux=3, steps=0)
    else:
        pr = problems.curved_lake(N=4, nel=10, seed=4, ripple=0.03, NumFlux=0, rotate_seed=5)
    s = Solver(pr, device_id=0)
    try:
        ref = s.rhs()
    finally:
        s.close()
    t64, t32 = _device_inputs(pr, torch)
    first = _noalloc_rhs(pr, t64, t32, torch)
    second = _noalloc_rhs(pr, t64, t32, torch)
    np.testing.assert_array_equal(first, ref)
    np.testing.assert_array_equal(second, ref)


def test_noalloc_rejects_meshes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    L = pkg.lib()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    ptr = ctypes.c_void_p(dummy.data_ptr())
    # 2^20 faces at N=4 need ~26M doubles of scratch, more than the fixed 2M
    rc = L.esdg_compute_rhs_noalloc(4, 1 << 19, 1 << 20, 0, 1, 9.81, 1e-4, *([ptr] * 17), ptr, None)
    assert rc == -1
    assert b"scratch" in L.esdg_last_error(None)


def test_noalloc_reports_bad_connectivity():
    """One ElemToEdge entry out of range: the entry point substitutes a safe
    face, still writes a finite right-hand side and returns ESDG_E_ARG."""
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    pr = problems.periodic_bump(N=3, nel=8, NumFlux=0, steps=0)
    t64, t32 = _device_inputs(pr, torch)
    t32[1][5] = pr.F + 7  # ElemToEdge of element 1, side 1: no such face
    rc, out = _noalloc_call(pr, t64, t32, torch)
    assert rc == -1
    assert b"connectivity" in pkg.lib().esdg_last_error(None)
    assert np.isfinite(out).all()
