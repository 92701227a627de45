"""Python mirror of the reference's ``deviceclass`` (include/deviceclass.h:28-138)
over the C ABI of libesdg_b200.so.  Method names, argument order and meaning
follow the reference; errors raise ``EsdgError`` carrying the engine's
status code and message (the reference aborts or throws instead).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lib as _lib
from .host import Problem, pd, pi

E_ARG, E_UNSUPPORTED, E_CUDA, E_NONFINITE, E_IO, E_NOMEM = -1, -2, -3, -4, -5, -6


class EsdgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _element_variants(L, fn, h, cap=8):
    chosen, count = ctypes.c_int(), ctypes.c_int()
    ms = (ctypes.c_float * cap)()
    ctas = (ctypes.c_int * cap)()
    rc = fn(h, ctypes.byref(chosen), ctypes.byref(count), ms, ctas, cap)
    if rc != 0:
        return None
    n = min(count.value, cap)
    return {"chosen": chosen.value, "count": count.value, "ms": [float(v) for v in ms[:n]],
            "ctas_per_sm": [int(v) for v in ctas[:n]]}


def _indicator_params(net):
    if net is None:
        raise ValueError("the learned indicator needs a network")
    P = np.ascontiguousarray(net.P, dtype=np.float32)
    return P.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), P.size, float(net.margin)


class DeviceClass:
    """One engine handle (one GPU, one mesh)."""

    def __init__(self, rank: int = 0, device_id: int = -1):
        self._L = _lib()
        h = ctypes.c_void_p()
        rc = self._L.esdg_deviceclass_create(rank, device_id, ctypes.byref(h))
        if rc != 0:
            raise EsdgError(rc, self._L.esdg_last_error(None).decode())
        self.h = h
        self._keep = []

    def _ok(self, rc):
        if rc != 0:
            raise EsdgError(rc, self._L.esdg_last_error(self.h).decode())

    # -- reference surface -------------------------------------------------
    def initDeviceVariables(self, N, Nelem, Nfaces, rank, rkSSP, NEpad, NEsurfpad, Nedgepad, NAvgPad, ES, Testcase,
                            epsilon_0, sigma_max, sigma_min, PosPresTOL, geomface, g_const, PositivityPreserving,
                            ArtificialViscosity, DiscBottom, h_0, PartialDry, FrictionTerms, CalcArrivalTimes,
                            CreateTimeSeries, CalcMaximumElevation):
        self._ok(self._L.esdg_init_device_variables(
            self.h, N, Nelem, Nfaces, rank, rkSSP, NEpad, NEsurfpad, Nedgepad, NAvgPad, ES, Testcase, epsilon_0,
            sigma_max, sigma_min, PosPresTOL, geomface, g_const, PositivityPreserving, ArtificialViscosity,
            DiscBottom, h_0, PartialDry, FrictionTerms, CalcArrivalTimes, CreateTimeSeries, CalcMaximumElevation))

    def copyDeviceVariables(self, PositivityPreserving, Nelem, GLw, normalsX, normalsY, Scal, y_xi, y_eta, x_xi,
                            x_eta, b, Bx, By, Dmat, Dstrong, Dhat, J, x_phy, y_phy, q, ElementSizes, gRK, Qt, VdmInv,
                            ElemEdgeMasterSlave, ElemEdgeOrientation, ElemToEdge, EdgeData, EdgeReversed):
        d = [_f64(a) for a in (GLw, normalsX, normalsY, Scal, y_xi, y_eta, x_xi, x_eta, b, Bx, By, Dmat, Dstrong,
                               Dhat, J, x_phy, y_phy, q, ElementSizes, gRK, Qt, VdmInv)]
        i = [_i32(a) for a in (ElemEdgeMasterSlave, ElemEdgeOrientation, ElemToEdge, EdgeData, EdgeReversed)]
        self._ok(self._L.esdg_copy_device_variables(self.h, PositivityPreserving, Nelem, *[pd(a) for a in d],
                                                    *[pi(a) for a in i]))

    def copyPartialDryData(self, DCentralFD, DforwardFD, DbackwardFD):
        """The difference matrices of the partial-dry volume term
        (deviceclass::copyPartialDryData; host.Basis.fd())."""
        d = [_f64(a) for a in (DCentralFD, DforwardFD, DbackwardFD)]
        self._ok(self._L.esdg_copy_partial_dry_data(self.h, *[pd(a) for a in d]))

    def buildDeviceKernels(self, KernelVersion, KernelVersionSTD, Testcase, FluxDifferencing, NumFlux, rkSSP,
                           ArtificialViscosity, PositivityPreserving, DiscBottom):
        self._ok(self._L.esdg_build_device_kernels(self.h, KernelVersion, KernelVersionSTD, Testcase,
                                                   FluxDifferencing, NumFlux, rkSSP, ArtificialViscosity,
                                                   PositivityPreserving, DiscBottom))

    def DGtimeloop(self, Nelem, Nfaces, rkA, rkB, rkC, globalMinEleSize, CFL, DFL, T, Testcase, ArtificialViscosity,
                   rkSSP, NumPlots, NumTimeChecks, g_const, PlotVar, EntropyPlot, PositivityPreserving, DiscBottom,
                   max_steps=0):
        A, B, C = _f64(rkA), _f64(rkB), _f64(rkC)
        t = ctypes.c_double()
        s = ctypes.c_int()
        self._ok(self._L.esdg_dg_timeloop(self.h, Nelem, Nfaces, len(A), pd(A), pd(B), pd(C), globalMinEleSize, CFL,
                                          DFL, T, Testcase, ArtificialViscosity, rkSSP, NumPlots, NumTimeChecks,
                                          g_const, PlotVar, EntropyPlot, PositivityPreserving, DiscBottom, max_steps,
                                          ctypes.byref(t), ctypes.byref(s)))
        return t.value, s.value

    def copy_q_to_host(self, q: np.ndarray):
        assert q.dtype == np.float64 and q.flags.c_contiguous
        self._ok(self._L.esdg_copy_q_to_host(self.h, pd(q)))
        return q

    def copy_q_from_host(self, q: np.ndarray):
        q = _f64(q)
        self._ok(self._L.esdg_copy_q_from_host(self.h, pd(q)))

    def bytesAllocated(self) -> int:
        return int(self._L.esdg_bytes_allocated(self.h))

    def freeOccaVars(self, rkSSP=0, PositivityPreserving=0, ArtificialViscosity=0):
        self._ok(self._L.esdg_free_occa_vars(self.h, rkSSP, PositivityPreserving, ArtificialViscosity))

    # -- engine extras ------------------------------------------------------
    def compute_rhs(self, K, ngl, AV=False):
        Qt = np.zeros(K * 3 * ngl * ngl)
        visc = np.zeros(K) if AV else None
        self._ok(self._L.esdg_compute_rhs(self.h, pd(Qt), pd(visc)))
        return (Qt, visc) if AV else Qt

    def copy_visc_to_host(self, K):
        v = np.zeros(K)
        self._ok(self._L.esdg_copy_visc_to_host(self.h, pd(v)))
        return v

    def copy_arrival_times(self, nodes: int):
        a = np.zeros(nodes)
        self._ok(self._L.esdg_copy_arrival_times(self.h, pd(a)))
        return a

    def copy_maximum_elevation(self, nodes: int):
        a = np.zeros(nodes)
        self._ok(self._L.esdg_copy_maximum_elevation(self.h, pd(a)))
        return a

    def set_stream(self, stream_ptr: int | None):
        self._ok(self._L.esdg_set_stream(self.h, ctypes.c_void_p(stream_ptr or 0)))

    def advance(self, nsteps: int, T: float):
        t = ctypes.c_double()
        s = ctypes.c_int()
        self._ok(self._L.esdg_advance(self.h, nsteps, T, ctypes.byref(t), ctypes.byref(s)))
        return t.value, s.value

    def profile_steps(self, nsteps: int):
        f = ctypes.c_double()
        e = ctypes.c_double()
        self._ok(self._L.esdg_profile_steps(self.h, nsteps, ctypes.byref(f), ctypes.byref(e)))
        return f.value, e.value

    def kernel_launches(self) -> int:
        return int(self._L.esdg_kernel_launches(self.h))

    def debug_bulk_wait_test(self, wait_limit_cycles: int, skip_tile: int):
        """Test hook of the element kernels' bounded bulk-copy waits: a
        shorter wait limit (clock cycles, 0: the default) and a tile whose
        copies are never issued (-1: none)."""
        self._ok(self._L.esdg_debug_bulk_wait_test(self.h, int(wait_limit_cycles), int(skip_tile)))

    def set_indicator(self, mode: int, net=None):
        """Indicator of the artificial-viscosity path: 0 the modal sensor and
        the viscous terms everywhere (the reference's path), 1 the modal
        sensor with the active set, 2 the learned indicator (`net`, an
        indicator.IndicatorNet) with the active set."""
        P, n, margin = _indicator_params(net) if mode >= 2 else (None, 0, 0.0)
        self._ok(self._L.esdg_set_indicator(self.h, mode, P, n, margin))

    def set_indicator_every_stage(self, every_stage: bool):
        """Learned indicator (modes 2, 3) at every RK stage (default) or once
        per step, its viscosity and active set kept for the step's stages."""
        self._ok(self._L.esdg_set_indicator_every_stage(self.h, int(bool(every_stage))))

    def indicator_stats(self, reset: bool = False):
        """Counts since the last reset: elements set to zero by the network,
        set to eps0 by the network, decided by the modal sensor, and with
        nonzero viscosity."""
        out = (ctypes.c_ulonglong * 4)()
        self._ok(self._L.esdg_indicator_stats(self.h, out, int(reset)))
        return dict(zip(("net_zero", "net_full", "modal", "viscous"), [int(v) for v in out]))

    def tuned_config(self):
        """Element-kernel occupancy chosen by the autotuner and the measured
        launch times of the variants (ms)."""
        c, st = ctypes.c_int(), ctypes.c_int()
        ms = (ctypes.c_float * 3)()
        rc = self._L.esdg_tuned_config(self.h, ctypes.byref(c), ctypes.byref(st), ms)
        return None if rc != 0 else {"ctas_per_sm": c.value, "stages": st.value,
                                     "variant_ms": [float(v) for v in ms]}

    def element_variants(self):
        """All element-kernel variants: the one in use, the autotuner's
        launch times (ms, 0 if not timed) and resident CTAs per SM (0: not
        available here); None before the tuning ran."""
        return _element_variants(self._L, self._L.esdg_element_variants, self.h)

    def set_element_variant(self, variant: int):
        """Fixes the element-kernel variant (-1: the autotuner's choice)."""
        self._ok(self._L.esdg_set_element_variant(self.h, int(variant)))

    def state_pointers(self):
        """Device addresses (q, b, VdmInv) of the engine's own buffers."""
        q, b, v = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        self._ok(self._L.esdg_state_pointers(self.h, ctypes.byref(q), ctypes.byref(b), ctypes.byref(v)))
        return q.value, b.value, v.value

    def close(self):
        if self.h is not None and self.h.value:
            self._L.esdg_deviceclass_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """main.cpp:925-1051 for one Problem: init, copy, build, time loop."""

    def __init__(self, prob: Problem, device_id: int = -1, q0=None, indicator: int = 0, net=None):
        self.prob = prob
        p, m, bs = prob.params, prob.mesh, prob.basis
        self.dc = DeviceClass(0, device_id)
        self.dc.initDeviceVariables(p.N, m.K, m.F, 0, p.rkSSP, p.NEpad, p.NEsurfpad, p.Nedgepad, p.NavgPad, p.ES,
                                    p.Testcase, p.epsilon_0, p.sigma_max, p.sigma_min, p.PosPresTOL, bs.geomface,
                                    p.g_const, p.PositivityPreserving, p.ArtificialViscosity, p.DiscBottom, p.h_0,
                                    p.PartialDryTreatment, 0, p.ArrivalTimings, 0, p.maximumElevation)
        zeros = np.zeros_like(prob.q0)
        self.dc.copyDeviceVariables(p.PositivityPreserving, m.K, bs.wGL, m.nx, m.ny, m.scal, m.y_xi, m.y_eta, m.x_xi,
                                    m.x_eta, prob.b, prob.Bx, prob.By, bs.D, bs.Dstrong, bs.Dhat, m.Jinv, m.x, m.y,
                                    prob.q0 if q0 is None else q0, prob.EleSizes, zeros, zeros, bs.VdmInv,
                                    m.MasterSlave, m.Orientation, m.ElemToEdge, m.EdgeData, m.EdgeReversed)
        if p.PartialDryTreatment:
            self.dc.copyPartialDryData(*(getattr(bs, "fd_mats", None) or bs.fd()))
        self.dc.buildDeviceKernels(99, 99, p.Testcase, p.FluxDifferencing, p.NumFlux, p.rkSSP, p.ArtificialViscosity,
                                   p.PositivityPreserving, p.DiscBottom)
        if indicator:
            self.dc.set_indicator(indicator, net)

    def run(self, T=None, max_steps=None):
        p, prob = self.prob.params, self.prob
        T = p.T if T is None else T
        ms = p.MaxSteps if max_steps is None else max_steps
        return self.dc.DGtimeloop(prob.K, prob.F, prob.rkA, prob.rkB, prob.rkC, prob.minEleSize, p.CFL, p.DFL, T,
                                  p.Testcase, p.ArtificialViscosity, p.rkSSP, 0, 0, p.g_const, 0, 0,
                                  p.PositivityPreserving, p.DiscBottom, ms)

    def q(self):
        return self.dc.copy_q_to_host(np.zeros_like(self.prob.q0))

    def rhs(self):
        return self.dc.compute_rhs(self.prob.K, self.prob.ngl, bool(self.prob.params.ArtificialViscosity))

    def arrival_times(self):
        return self.dc.copy_arrival_times(self.prob.K * self.prob.ngl ** 2)

    def maximum_elevation(self):
        return self.dc.copy_maximum_elevation(self.prob.K * self.prob.ngl ** 2)

    def close(self):
        self.dc.close()
