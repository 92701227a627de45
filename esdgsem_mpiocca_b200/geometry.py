"""Curvilinear element geometry built on the device (esdg_geometry_device):
nodal coordinates by the transfinite map of the element's boundary curves,
collocation metric terms, Jacobian and side normals -- the same bits as the
host set-up (src/Mesh.cpp:1000-1081, 1619-1650, 1667-1808).

`element_curves` exports a host mesh's corners, curve flags and side samples
(the ISM-V2 representation); `device_geometry` builds the geometry from them
on the GPU; `face_normals` gathers the face-major normals the device layer
takes (main.cpp:650-716: the left element's side).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import lib as _lib
from .host import _check, pd, pi


def element_curves(make, N):
    """(curve_order, corners [K][4][2], curved [K][4], curves [K][4][m+1][2])
    of the mesh that `make(out_handle_ptr)` constructs (e.g. a call of
    esdg_mesh_mapped or esdg_mesh_read_ism2)."""
    L = _lib()
    h = ctypes.c_void_p()
    _check(make(ctypes.byref(h)), "mesh construction")
    try:
        K, F = ctypes.c_int(), ctypes.c_int()
        _check(L.esdg_mesh_sizes(h, ctypes.byref(K), ctypes.byref(F)), "esdg_mesh_sizes")
        m = ctypes.c_int()
        _check(L.esdg_mesh_element_curves(h, ctypes.byref(m), None, None, None), "esdg_mesh_element_curves")
        K, m = K.value, m.value
        corners = np.zeros((K, 4, 2))
        curved = np.zeros((K, 4), dtype=np.int32)
        curves = np.zeros((K, 4, m + 1, 2))
        _check(L.esdg_mesh_element_curves(h, ctypes.byref(ctypes.c_int()), pd(corners), pi(curved), pd(curves)),
               "esdg_mesh_element_curves")
    finally:
        L.esdg_mesh_free(h)
    return m, corners, curved, curves


def device_geometry(N, curve_order, corners, curved, curves, stream=None):
    """Geometry of every element, computed on the current CUDA device:
    dict of torch tensors x, y, x_xi, x_eta, y_xi, y_eta, J [K*(N+1)^2] and
    nx_side, ny_side, scal_side [K*4*(N+1)]."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    K = int(corners.shape[0])
    n2 = (N + 1) ** 2
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)  # noqa: E731
    c, g, v = t(corners, np.float64), t(curved, np.int32), t(curves, np.float64)
    out = {k: torch.empty(K * n2, dtype=torch.float64, device=dev)
           for k in ("x", "y", "x_xi", "x_eta", "y_xi", "y_eta", "J")}
    for k in ("nx_side", "ny_side", "scal_side"):
        out[k] = torch.empty(K * 4 * (N + 1), dtype=torch.float64, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    vp = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    rc = _lib().esdg_geometry_device(N, K, int(curve_order), vp(c), vp(g), vp(v), vp(out["x"]), vp(out["y"]),
                                     vp(out["x_xi"]), vp(out["x_eta"]), vp(out["y_xi"]), vp(out["y_eta"]),
                                     vp(out["J"]), vp(out["nx_side"]), vp(out["ny_side"]), vp(out["scal_side"]),
                                     ctypes.c_void_p(s))
    if rc != 0:
        raise RuntimeError(f"esdg_geometry_device failed ({rc}): {_lib().esdg_last_error(None).decode()}")
    return out


def face_normals(side_array, EdgeData, N):
    """Face-major [F*(N+1)] values of a [K*4*(N+1)] side array: each face
    takes its left element's side (main.cpp:650-716)."""
    n = N + 1
    ed = np.asarray(EdgeData).reshape(-1, 8)
    base = (ed[:, 0].astype(np.int64) * 4 + ed[:, 2]) * n
    idx = base[:, None] + np.arange(n)[None, :]
    return np.asarray(side_array)[idx].reshape(-1)
