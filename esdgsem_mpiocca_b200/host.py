"""Host-side set-up in the reference's order (main.cpp:270-921): basis,
mesh, packed connectivity, bathymetry gradient, element sizes, RK tables.
All numbers come from libesdg_b200.so's set-up entry points (C++); this
module only owns the numpy buffers.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import lib as _lib

_PD = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)


def pd(a):
    return None if a is None else a.ctypes.data_as(_PD)


def pi(a):
    return None if a is None else a.ctypes.data_as(_PI)


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


@dataclass
class Basis:
    N: int
    xGL: np.ndarray
    wGL: np.ndarray
    xG: np.ndarray
    wG: np.ndarray
    D: np.ndarray       # flux-differencing form
    D0: np.ndarray
    Dstrong: np.ndarray
    Dhat: np.ndarray
    VdmInv: np.ndarray

    @staticmethod
    def build(N: int, flux_differencing: int = 1) -> "Basis":
        n = N + 1
        arr = [np.zeros(n) for _ in range(4)] + [np.zeros(n * n) for _ in range(5)]
        _check(_lib().esdg_basis(N, flux_differencing, *[pd(a) for a in arr]), "esdg_basis")
        return Basis(N, *arr)

    @property
    def geomface(self) -> float:
        """1/w_0 (main.cpp:921)."""
        return 1.0 / self.wGL[0]

    def fd(self):
        """Central, forward and backward difference matrices [n*n] of the
        partial-dry treatment (src/basis.cpp:190-229)."""
        n2 = (self.N + 1) ** 2
        out = [np.zeros(n2) for _ in range(3)]
        _check(_lib().esdg_basis_fd(self.N, *[pd(a) for a in out]), "esdg_basis_fd")
        return tuple(out)


@dataclass
class MeshArrays:
    N: int
    K: int
    F: int
    x: np.ndarray
    y: np.ndarray
    x_xi: np.ndarray
    x_eta: np.ndarray
    y_xi: np.ndarray
    y_eta: np.ndarray
    Jinv: np.ndarray
    nx: np.ndarray
    ny: np.ndarray
    scal: np.ndarray
    b: np.ndarray
    EdgeData: np.ndarray
    EdgeReversed: np.ndarray
    ElemToEdge: np.ndarray
    MasterSlave: np.ndarray
    Orientation: np.ndarray


def _pack(handle, N) -> MeshArrays:
    L = _lib()
    K = ctypes.c_int()
    F = ctypes.c_int()
    _check(L.esdg_mesh_sizes(handle, ctypes.byref(K), ctypes.byref(F)), "esdg_mesh_sizes")
    K, F = K.value, F.value
    n = N + 1
    nn = K * n * n
    d = {k: np.zeros(nn) for k in ("x", "y", "x_xi", "x_eta", "y_xi", "y_eta", "Jinv", "b")}
    for k in ("nx", "ny", "scal"):
        d[k] = np.zeros(F * n)
    ED = np.zeros(F * 8, dtype=np.int32)
    ER = np.zeros(F, dtype=np.int32)
    E2E = np.zeros(K * 4, dtype=np.int32)
    MS = np.zeros(K * 4, dtype=np.int32)
    OR = np.zeros(K * 4, dtype=np.int32)
    _check(L.esdg_mesh_pack(handle, pd(d["x"]), pd(d["y"]), pd(d["x_xi"]), pd(d["x_eta"]), pd(d["y_xi"]),
                            pd(d["y_eta"]), pd(d["Jinv"]), pd(d["nx"]), pd(d["ny"]), pd(d["scal"]), pd(d["b"]),
                            pi(ED), pi(ER), pi(E2E), pi(MS), pi(OR)), "esdg_mesh_pack")
    return MeshArrays(N, K, F, EdgeData=ED, EdgeReversed=ER, ElemToEdge=E2E, MasterSlave=MS, Orientation=OR, **d)


def _with_handle(make, N, write_path=None) -> MeshArrays:
    L = _lib()
    h = ctypes.c_void_p()
    rc = make(ctypes.byref(h))
    _check(rc, "mesh construction")
    try:
        if write_path:
            _check(L.esdg_mesh_write_ism2(h, str(write_path).encode()), "esdg_mesh_write_ism2")
        return _pack(h, N)
    finally:
        L.esdg_mesh_free(h)


def mesh_cartesian(N, xL, xR, yL, yR, NX, NY, periodic_rows=False, periodic_cols=False) -> MeshArrays:
    """Mesh::GenerateMesh (src/Mesh.cpp:316-696)."""
    return _with_handle(lambda out: _lib().esdg_mesh_cartesian(N, xL, xR, yL, yR, NX, NY, int(periodic_rows),
                                                               int(periodic_cols), out), N)


def mesh_mapped(N, xL, xR, yL, yR, NX, NY, amp=0.03, curve_order=None, rotate_seed=0, write_path=None) -> MeshArrays:
    """Curved structured mesh, every side an order-m boundary curve (ISM-V2 form)."""
    m = curve_order if curve_order is not None else max(N, 4)
    return _with_handle(lambda out: _lib().esdg_mesh_mapped(N, xL, xR, yL, yR, NX, NY, amp, m, rotate_seed, out), N,
                        write_path)


def mesh_read(N, path, read_bottom=False, convert_km=False) -> MeshArrays:
    """Mesh::ReadMesh (src/Mesh.cpp:698-1503)."""
    return _with_handle(lambda out: _lib().esdg_mesh_read_ism2(N, str(path).encode(), int(read_bottom),
                                                               int(convert_km), out), N)


def bottom_derivatives(mesh: MeshArrays, basis: Basis, b: np.ndarray):
    """SW2D::CalcBDerivatives (src/SW2D.cpp:1048-1105)."""
    Bx = np.zeros_like(b)
    By = np.zeros_like(b)
    _check(_lib().esdg_bottom_derivatives(mesh.K, mesh.N, pd(basis.D0), pd(b), pd(mesh.y_eta), pd(mesh.y_xi),
                                          pd(mesh.x_eta), pd(mesh.x_xi), pd(mesh.Jinv), pd(Bx), pd(By)),
           "esdg_bottom_derivatives")
    return Bx, By


def element_sizes(mesh: MeshArrays, basis: Basis):
    """basis::calcElementSizes (src/basis.cpp:939-966)."""
    es = np.zeros(mesh.K)
    mn = ctypes.c_double()
    _check(_lib().esdg_element_sizes(mesh.K, mesh.N, pd(basis.wGL), pd(mesh.Jinv), pd(es), ctypes.byref(mn)),
           "esdg_element_sizes")
    return es, mn.value


def rk_coefficients(order: int, ssp: int):
    """RungeKutta::RungeKutta (src/RungeKutta.cpp:18-90)."""
    A, B, C = np.zeros(8), np.zeros(8), np.zeros(8)
    s = ctypes.c_int()
    _check(_lib().esdg_rk_coefficients(order, ssp, pd(A), pd(B), pd(C), ctypes.byref(s)), "esdg_rk_coefficients")
    return A[: s.value].copy(), B[: s.value].copy(), C[: s.value].copy()


def diagnostics(mesh: MeshArrays, basis: Basis, q, qref=None, b=None, g=9.81):
    """L2 / Linf error, total mass and entropy (src/basis.cpp:874-1111)."""
    L2, Li = np.zeros(3), np.zeros(3)
    m = ctypes.c_double()
    S = ctypes.c_double()
    _check(_lib().esdg_diagnostics(mesh.K, mesh.N, pd(basis.wGL), pd(mesh.Jinv), pd(q), pd(qref), pd(b), g, pd(L2),
                                   pd(Li), ctypes.byref(m), ctypes.byref(S)), "esdg_diagnostics")
    return {"L2": L2, "Linf": Li, "mass": m.value, "entropy": S.value}


@dataclass
class Params:
    """The input.dat parameters the hot path reads (src/ReadInput.cpp:155-247)."""
    N: int = 3
    CFL: float = 0.4
    DFL: float = 0.1
    T: float = 1.0
    g_const: float = 9.81
    ArtificialViscosity: int = 0
    PositivityPreserving: int = 0
    PosPresTOL: float = 1e-4
    epsilon_0: float = 0.1
    sigma_min: float = -16.0
    sigma_max: float = -12.0
    Testcase: int = 0
    ES: int = 1
    NumFlux: int = 0
    FluxDifferencing: int = 1
    rkOrder: int = 4
    rkSSP: int = 0
    NEpad: int = 4
    NEsurfpad: int = 16
    Nedgepad: int = 16
    NavgPad: int = 10
    DiscBottom: int = 0
    PartialDryTreatment: int = 0
    MaxSteps: int = 0
    # analysis outputs (input.dat lines ArrivalTimings / maximumElevation)
    # and the still-water level h_0 they are measured from
    ArrivalTimings: int = 0
    maximumElevation: int = 0
    h_0: float = 0.0


@dataclass
class Problem:
    """Everything copyDeviceVariables and DGtimeloop receive."""
    params: Params
    basis: Basis
    mesh: MeshArrays
    b: np.ndarray
    Bx: np.ndarray
    By: np.ndarray
    q0: np.ndarray
    EleSizes: np.ndarray
    minEleSize: float
    rkA: np.ndarray
    rkB: np.ndarray
    rkC: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def K(self):
        return self.mesh.K

    @property
    def F(self):
        return self.mesh.F

    @property
    def ngl(self):
        return self.params.N + 1

    def dofs(self) -> int:
        return self.mesh.K * self.ngl * self.ngl


def make_problem(params: Params, mesh: MeshArrays, b: np.ndarray, q0: np.ndarray, meta=None) -> Problem:
    basis = Basis.build(params.N, params.FluxDifferencing)
    b = np.ascontiguousarray(b, dtype=np.float64)
    Bx, By = bottom_derivatives(mesh, basis, b)
    es, mn = element_sizes(mesh, basis)
    A, B, C = rk_coefficients(params.rkOrder, params.rkSSP)
    return Problem(params, basis, mesh, b, Bx, By, np.ascontiguousarray(q0, dtype=np.float64), es, mn, A, B, C,
                   meta or {})
