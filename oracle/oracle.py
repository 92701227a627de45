"""ORACLE -- test infrastructure only.

ctypes binding of oracle/_build/libesdg_oracle.so, the plain-C restatement of
the reference kernels and time loop (oracle/esdg_oracle.c).  Imported only by
tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference legs;
the engine never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_build", "libesdg_oracle.so")

_PD = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)


class _Geom(ctypes.Structure):
    _fields_ = [(n, _PD) for n in ("Jinv", "Yxi", "Yeta", "Xxi", "Xeta", "Bx", "By", "B", "nx", "ny", "scal", "D",
                                   "Dstrong", "Dhat", "VdmInv", "GLw", "EleSizes")] + \
               [(n, _PI) for n in ("EdgeData", "EdgeReversed", "ElemToEdge", "MasterSlave", "Orientation")] + \
               [(n, _PD) for n in ("DcFD", "DfFD", "DbFD")] + [("PD", ctypes.c_int)] + \
               [(n, _PD) for n in ("X", "Y")] + [("Testcase", ctypes.c_int)] + \
               [(n, _PD) for n in ("ArrivalTimes", "MaxElevation")] + [("h0", ctypes.c_double)]


_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        src = os.path.join(HERE, "esdg_oracle.c")
        if not os.path.exists(SO) or os.path.getmtime(SO) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(SO)
        G = ctypes.POINTER(_Geom)
        D, I = ctypes.c_double, ctypes.c_int
        L.oracle_rhs.argtypes = [I, I, I, D, D, I, I, G, _PD, _PD, _PD]
        L.oracle_timeloop.argtypes = [I, I, I, G, _PD, D, D, I, I, I, _PD, _PD, _PD, I, I, I, D, D, D, D, D, D, D, I,
                                      _PD, _PI, _PD, _PD]
        L.oracle_timeloop.restype = I
        L.oracle_lambda_max.argtypes = [I, I, D, D, _PD, _PD]
        L.oracle_pos_pres.argtypes = [I, I, D, _PD, _PD, _PD, _PD]
        L.oracle_shock_capturing.argtypes = [I, I, D, D, D, _PD, _PD, _PD, _PD]
        L.oracle_viscous_rhs.argtypes = [I, I, I, G, D, _PD, _PD, _PD]
        _LIB = L
    return _LIB


def _p(a, t=_PD):
    return a.ctypes.data_as(t)


class OracleProblem:
    """Borrowed view of a host Problem (esdgsem_mpiocca_b200.host.Problem)."""

    def __init__(self, prob):
        self.prob = prob
        m, bs = prob.mesh, prob.basis
        self._arrs = dict(Jinv=m.Jinv, Yxi=m.y_xi, Yeta=m.y_eta, Xxi=m.x_xi, Xeta=m.x_eta, Bx=prob.Bx, By=prob.By,
                          B=prob.b, nx=m.nx, ny=m.ny, scal=m.scal, D=bs.D, Dstrong=bs.Dstrong, Dhat=bs.Dhat,
                          VdmInv=bs.VdmInv, GLw=bs.wGL, EleSizes=prob.EleSizes)
        self._ints = dict(EdgeData=m.EdgeData, EdgeReversed=m.EdgeReversed, ElemToEdge=m.ElemToEdge,
                          MasterSlave=m.MasterSlave, Orientation=m.Orientation)
        for k, v in self._arrs.items():
            assert v.dtype == np.float64 and v.flags.c_contiguous, k
        for k, v in self._ints.items():
            assert v.dtype == np.int32 and v.flags.c_contiguous, k
        pd = int(getattr(prob.params, "PartialDryTreatment", 0))
        fd = getattr(prob.basis, "fd_mats", None) or prob.basis.fd()
        self._fd = [np.ascontiguousarray(a, dtype=np.float64) for a in fd]
        self._xy = [np.ascontiguousarray(a, dtype=np.float64) for a in (m.x, m.y)]
        self.g = _Geom(**{k: _p(v) for k, v in self._arrs.items()}, **{k: _p(v, _PI) for k, v in self._ints.items()},
                       DcFD=_p(self._fd[0]), DfFD=_p(self._fd[1]), DbFD=_p(self._fd[2]), PD=pd,
                       X=_p(self._xy[0]), Y=_p(self._xy[1]), Testcase=int(prob.params.Testcase),
                       h0=float(getattr(prob.params, "h_0", 0.0)))

    def rhs(self, q):
        p = self.prob.params
        q = np.ascontiguousarray(q, dtype=np.float64)
        Qt = np.zeros_like(q)
        lib().oracle_rhs(p.N, self.prob.K, self.prob.F, p.g_const, p.PosPresTOL, p.ES, p.NumFlux,
                         ctypes.byref(self.g), _p(q), _p(Qt), None)
        if p.ArtificialViscosity:
            visc = np.zeros(self.prob.K)
            lib().oracle_shock_capturing(p.N, self.prob.K, p.epsilon_0, p.sigma_min, p.sigma_max, _p(q),
                                         _p(self.prob.b), _p(self.prob.basis.VdmInv), _p(visc))
            lib().oracle_viscous_rhs(p.N, self.prob.K, self.prob.F, ctypes.byref(self.g), p.PosPresTOL, _p(q),
                                     _p(visc), _p(Qt))
            return Qt, visc
        return Qt

    def run(self, q=None, T=None, max_steps=None, log_dt=False):
        p = self.prob.params
        q = np.array(self.prob.q0 if q is None else q, dtype=np.float64, copy=True)
        T = p.T if T is None else T
        ms = p.MaxSteps if max_steps is None else max_steps
        t = ctypes.c_double()
        s = ctypes.c_int()
        dts = np.zeros(max(ms, 1)) if (log_dt and ms > 0) else None
        visc = np.zeros(self.prob.K) if p.ArtificialViscosity else None
        A, B, C = (np.ascontiguousarray(v, dtype=np.float64) for v in (self.prob.rkA, self.prob.rkB, self.prob.rkC))
        nodes = self.prob.K * (p.N + 1) ** 2
        at = np.full(nodes, 1000.0) if getattr(p, "ArrivalTimings", 0) else None
        me = np.zeros(nodes) if getattr(p, "maximumElevation", 0) else None
        self.g.ArrivalTimes = None if at is None else _p(at)
        self.g.MaxElevation = None if me is None else _p(me)
        rc = lib().oracle_timeloop(p.N, self.prob.K, self.prob.F, ctypes.byref(self.g), _p(q), p.g_const,
                                   p.PosPresTOL, p.ES, p.NumFlux, len(A), _p(A), _p(B), _p(C), p.rkSSP,
                                   p.ArtificialViscosity, p.PositivityPreserving, p.epsilon_0, p.sigma_min,
                                   p.sigma_max, self.prob.minEleSize, p.CFL, p.DFL, T, ms, ctypes.byref(t),
                                   ctypes.byref(s), None if dts is None else _p(dts),
                                   None if visc is None else _p(visc))
        self.g.ArrivalTimes = self.g.MaxElevation = None
        assert rc == 0
        out = {"q": q, "t": t.value, "steps": s.value}
        if at is not None:
            out["ArrivalTimings"] = at
        if me is not None:
            out["MaximumElevation"] = me
        if dts is not None:
            out["dt"] = dts[: s.value]
        if visc is not None:
            out["visc"] = visc
        return out

    def lambda_max(self, q):
        p = self.prob.params
        out = ctypes.c_double()
        q = np.ascontiguousarray(q, dtype=np.float64)
        lib().oracle_lambda_max(p.N, self.prob.K, p.g_const, p.PosPresTOL, _p(q), ctypes.byref(out))
        return out.value


def set_threads(n: int):
    os.environ["OMP_NUM_THREADS"] = str(n)
