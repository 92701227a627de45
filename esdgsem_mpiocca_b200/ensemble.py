"""Batched ensemble engine (arena) over the C ABI: many independent instances
of one polynomial degree advance together, every kernel launch covering all
of them, each instance with its own time step from its own CFL reduction,
end time and step cap.  Instances can be added and removed between steps
(continuous batching); the step graph stays the same.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lib as _lib
from .deviceclass import EsdgError
from .host import Problem, pd, pi


class Ensemble:
    def __init__(self, N, max_instances, K_capacity, F_capacity, NumFlux=0, ES=1, g_const=9.81, PosPresTOL=1e-4,
                 ArtificialViscosity=0, epsilon_0=0.0, sigma_max=0.0, sigma_min=0.0, PositivityPreserving=0,
                 rkOrder=4, rkSSP=0, device_id=-1):
        self._L = _lib()
        h = ctypes.c_void_p()
        rc = self._L.esdg_ensemble_create(device_id, N, max_instances, K_capacity, F_capacity, NumFlux, ES, g_const,
                                          PosPresTOL, ArtificialViscosity, epsilon_0, sigma_max, sigma_min,
                                          PositivityPreserving, rkOrder, rkSSP, ctypes.byref(h))
        if rc != 0:
            raise EsdgError(rc, self._L.esdg_ensemble_last_error(None).decode())
        self.h = h
        self.N = N
        self.sizes = {}

    @staticmethod
    def for_problems(probs, max_instances=None, slack=1.0, **kw):
        p0 = probs[0].params
        K = int(sum(p.K for p in probs) * slack)
        F = int(sum(p.F for p in probs) * slack)
        args = dict(NumFlux=p0.NumFlux, ES=p0.ES, g_const=p0.g_const, PosPresTOL=p0.PosPresTOL,
                    ArtificialViscosity=p0.ArtificialViscosity, epsilon_0=p0.epsilon_0, sigma_max=p0.sigma_max,
                    sigma_min=p0.sigma_min, PositivityPreserving=p0.PositivityPreserving, rkOrder=p0.rkOrder,
                    rkSSP=p0.rkSSP)
        args.update(kw)
        return Ensemble(p0.N, max_instances or len(probs), K, F, **args)

    def _ok(self, rc):
        if rc != 0:
            raise EsdgError(rc, self._L.esdg_ensemble_last_error(self.h).decode())

    def add(self, prob: Problem, T=None, max_steps=None, q0=None) -> int:
        m, p = prob.mesh, prob.params
        q = np.ascontiguousarray(prob.q0 if q0 is None else q0, dtype=np.float64)
        out = ctypes.c_int()
        self._ok(self._L.esdg_ensemble_add(
            self.h, m.K, m.F, pd(m.nx), pd(m.ny), pd(m.scal), pd(m.y_xi), pd(m.y_eta), pd(m.x_xi), pd(m.x_eta),
            pd(prob.b), pd(prob.Bx), pd(prob.By), pd(m.Jinv), pd(q), pd(prob.EleSizes), pi(m.MasterSlave),
            pi(m.Orientation), pi(m.ElemToEdge), pi(m.EdgeData), p.T if T is None else T,
            p.MaxSteps if max_steps is None else max_steps, prob.minEleSize, p.CFL, p.DFL, ctypes.byref(out)))
        self.sizes[out.value] = q.size
        return out.value

    def remove(self, i: int):
        self._ok(self._L.esdg_ensemble_remove(self.h, i))
        self.sizes.pop(i, None)

    def advance(self, nsteps: int):
        self._ok(self._L.esdg_ensemble_advance(self.h, nsteps))

    def launch(self, nsteps: int):
        """advance() without waiting; sync() waits and refreshes status."""
        self._ok(self._L.esdg_ensemble_launch(self.h, nsteps))

    def sync(self):
        self._ok(self._L.esdg_ensemble_sync(self.h))

    def status(self, i: int):
        t, s, d, st = ctypes.c_double(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._ok(self._L.esdg_ensemble_status(self.h, i, ctypes.byref(t), ctypes.byref(s), ctypes.byref(d),
                                              ctypes.byref(st)))
        return {"t": t.value, "steps": s.value, "done": bool(d.value), "status": st.value}

    def q(self, i: int):
        out = np.zeros(self.sizes[i])
        self._ok(self._L.esdg_ensemble_copy_q(self.h, i, pd(out)))
        return out

    def free_capacity(self):
        k, f, s = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._ok(self._L.esdg_ensemble_free_capacity(self.h, ctypes.byref(k), ctypes.byref(f), ctypes.byref(s)))
        return k.value, f.value, s.value

    def bytes(self) -> int:
        return int(self._L.esdg_ensemble_bytes(self.h))

    def kernel_launches(self) -> int:
        return int(self._L.esdg_ensemble_kernel_launches(self.h))

    def set_indicator(self, mode: int, net=None):
        """0: modal sensor and viscous terms everywhere (the reference's
        path); 1: modal sensor with the active set; 2: the learned indicator
        (indicator.IndicatorNet) with the active set."""
        from .deviceclass import _indicator_params
        P, n, margin = _indicator_params(net) if mode >= 2 else (None, 0, 0.0)
        self._ok(self._L.esdg_ensemble_set_indicator(self.h, mode, P, n, margin))

    def set_indicator_every_stage(self, every_stage: bool):
        """Learned indicator at every RK stage (default) or once per step."""
        self._ok(self._L.esdg_ensemble_set_indicator_every_stage(self.h, int(bool(every_stage))))

    def indicator_stats(self, reset: bool = False):
        out = (ctypes.c_ulonglong * 4)()
        self._ok(self._L.esdg_ensemble_indicator_stats(self.h, out, int(reset)))
        return dict(zip(("net_zero", "net_full", "modal", "viscous"), [int(v) for v in out]))

    def element_variants(self):
        from .deviceclass import _element_variants
        return _element_variants(self._L, self._L.esdg_ensemble_element_variants, self.h)

    def set_element_variant(self, variant: int):
        """Fixes the element-kernel variant (-1: the autotuner's choice)."""
        self._ok(self._L.esdg_ensemble_set_element_variant(self.h, int(variant)))

    def set_stream(self, stream_ptr):
        self._ok(self._L.esdg_ensemble_set_stream(self.h, ctypes.c_void_p(stream_ptr or 0)))

    def run_until_done(self, ids=None, chunk=8, max_launches=10 ** 7):
        ids = list(self.sizes) if ids is None else list(ids)
        n = 0
        while n < max_launches:
            self.advance(chunk)
            n += chunk
            if all(self.status(i)["done"] for i in ids):
                return n
        raise RuntimeError("ensemble did not finish")

    def close(self):
        if self.h is not None and self.h.value:
            self._L.esdg_ensemble_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
