"""Sea-surface uplift of a rectangular fault (Okada 1985, vertical surface
displacement from strike-slip and dip-slip dislocations), restated from
src/okada.cpp:33-249 of the reference.

Two front-ends share the dislocation core:
  * uplift_mercator: the reference's own geometry (src/okada.cpp:33-195):
    node coordinates in kilometres of a Mercator projection of lon/lat, the
    fault given by its epicentre (lon, lat), depth, length, width, strike,
    slip (rake) and dip angles and dislocation, uplift applied inside the
    reference's lon/lat-aligned box around the epicentre;
  * uplift_cartesian: the same dislocation model on plane coordinates in
    metres (for synthetic scenarios on a Cartesian square), applied inside a
    box of half-size 1.5 * max(length, width) around the centroid.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

EARTH_RADIUS = 6.378e6  # m, as src/okada.cpp:44


def _terms(x2, y1, y2, dp, dd):
    sn = np.sin(dp)
    cs = np.cos(dp)
    q = x2 * sn - dd * cs
    d_bar = y2 * sn - q * cs
    r = np.sqrt(y1 * y1 + y2 * y2 + q * q)
    xx = np.sqrt(y1 * y1 + q * q)
    return sn, cs, q, d_bar, r, xx


def strike_slip(x2, y1, y2, dp, dd):
    """f of the strike-slip component at one corner (src/okada.cpp:196-222)."""
    sn, cs, q, d_bar, r, xx = _terms(x2, y1, y2, dp, dd)
    a4 = 0.5 * 1.0 / cs * (np.log(r + d_bar) - sn * np.log(r + y2))
    return -(d_bar * q / r / (r + y2) + q * sn / (r + y2) + a4 * sn) / (2.0 * np.pi)


def dip_slip(x2, y1, y2, dp, dd):
    """f of the dip-slip component at one corner (src/okada.cpp:224-249)."""
    sn, cs, q, d_bar, r, xx = _terms(x2, y1, y2, dp, dd)
    a5 = 0.5 * 2 / cs * np.arctan((y2 * (xx + q * cs) + xx * (r + xx) * sn) / y1 / (r + xx) / cs)
    return -(d_bar * q / r / (r + y1) + sn * np.arctan(y1 * y2 / q / r) - a5 * sn * cs) / (2.0 * np.pi)


def _dislocation(x1, x2, hh, halfl, w, ang_l, ds, dd):
    """Vertical displacement from the four corners (src/okada.cpp:160-181)."""
    cs, sn = np.cos(ang_l), np.sin(ang_l)
    p = x2 * cs + hh * sn
    f1 = strike_slip(x2, x1 + halfl, p, ang_l, hh)
    f2 = strike_slip(x2, x1 + halfl, p - w, ang_l, hh)
    f3 = strike_slip(x2, x1 - halfl, p, ang_l, hh)
    f4 = strike_slip(x2, x1 - halfl, p - w, ang_l, hh)
    g1 = dip_slip(x2, x1 + halfl, p, ang_l, hh)
    g2 = dip_slip(x2, x1 + halfl, p - w, ang_l, hh)
    g3 = dip_slip(x2, x1 - halfl, p, ang_l, hh)
    g4 = dip_slip(x2, x1 - halfl, p - w, ang_l, hh)
    return (f1 - f2 - f3 + f4) * ds + (g1 - g2 - g3 + g4) * dd


@dataclass
class Fault:
    """Rectangular fault.  For uplift_mercator x0/y0 are the epicentre's
    longitude/latitude in degrees; for uplift_cartesian the centroid in metres.
    depth, length, width, slip in metres; angles in degrees."""
    x0: float
    y0: float
    depth: float
    length: float
    width: float
    strike: float
    rake: float
    dip: float
    slip: float


def uplift_mercator(x_km, y_km, f: Fault):
    """Uplift (in kilometres, as added to h by src/okada.cpp:183) at nodes
    given in Mercator kilometres."""
    rad = np.pi / 180.0
    R = EARTH_RADIUS
    x0m = f.x0 * R * np.pi / 180.0
    y0m = R * np.arcsinh(np.tan(f.y0 / 180.0 * np.pi))
    xlower, xupper, ylower, yupper = x0m - f.length, x0m + f.length, y0m - f.width, y0m + f.width
    xo = (xlower / R) * (180.0 / np.pi)
    yo = np.arctan(np.sinh(ylower / R)) * (180.0 / np.pi)
    ang_l, ang_r, ang_t = rad * f.dip, rad * f.rake, rad * f.strike
    halfl = 0.5 * f.length
    hh = f.depth + f.width * np.sin(ang_l)
    del_x = f.width * np.cos(ang_l) * np.cos(ang_t)
    del_y = f.width * np.cos(ang_l) * np.sin(ang_t)
    yl = R * (f.y0 - yo) * rad - del_y
    ds, dd = f.slip * np.cos(ang_r), f.slip * np.sin(ang_r)
    xloc = np.asarray(x_km, dtype=np.float64) * 1000.0
    yloc = np.asarray(y_km, dtype=np.float64) * 1000.0
    inside = (xloc >= xlower) & (xloc <= xupper) & (yloc >= ylower) & (yloc <= yupper)
    out = np.zeros_like(xloc)
    if not inside.any():
        return out
    xd = (xloc[inside] / R) * (180.0 / np.pi)
    yd = np.arctan(np.sinh(yloc[inside] / R)) * (180.0 / np.pi)
    xl = R * np.cos(rad * yd) * (f.x0 - xo) * rad + del_x
    yy = R * (yd - yo) * rad
    xx = R * np.cos(rad * yd) * (xd - xo) * rad
    x1 = (xx - xl) * np.sin(ang_t) + (yy - yl) * np.cos(ang_t)
    x2 = -((xx - xl) * np.cos(ang_t) - (yy - yl) * np.sin(ang_t))
    out[inside] = _dislocation(x1, x2, hh, halfl, f.width, ang_l, ds, dd) / 1000.0
    return out


def uplift_cartesian(x_m, y_m, f: Fault):
    """Uplift in metres at nodes in metres of a plane; the fault centroid is
    (f.x0, f.y0) and the epicentre offset of the reference (del_x, del_y)
    is applied as there."""
    rad = np.pi / 180.0
    ang_l, ang_r, ang_t = rad * f.dip, rad * f.rake, rad * f.strike
    halfl = 0.5 * f.length
    hh = f.depth + f.width * np.sin(ang_l)
    del_x = f.width * np.cos(ang_l) * np.cos(ang_t)
    del_y = f.width * np.cos(ang_l) * np.sin(ang_t)
    ds, dd = f.slip * np.cos(ang_r), f.slip * np.sin(ang_r)
    x = np.asarray(x_m, dtype=np.float64)
    y = np.asarray(y_m, dtype=np.float64)
    reach = 1.5 * max(f.length, f.width)
    inside = (np.abs(x - f.x0) <= reach) & (np.abs(y - f.y0) <= reach)
    out = np.zeros_like(x)
    if not inside.any():
        return out
    dx = (x[inside] - f.x0) - del_x
    dy = (y[inside] - f.y0) + del_y
    x1 = dx * np.sin(ang_t) + dy * np.cos(ang_t)
    x2 = -(dx * np.cos(ang_t) - dy * np.sin(ang_t))
    with np.errstate(divide="ignore", invalid="ignore"):
        u = _dislocation(x1, x2, hh, halfl, f.width, ang_l, ds, dd)
    out[inside] = np.where(np.isfinite(u), u, 0.0)
    return out


def uplift_device(x, y, f: Fault, mercator=False, out=None, add=False, stream=None):
    """The uplift computed on the GPU (esdg_okada_uplift: the same formulas
    in CUDA) at device points x, y (torch float64 tensors on the current
    device); returns `out` (a new tensor unless given; with add the uplift
    is added to it).  mercator selects uplift_mercator's geometry (x, y in
    Mercator km), else uplift_cartesian's (metres)."""
    import ctypes
    import torch
    from . import lib as _lib
    x = x.contiguous()
    y = y.contiguous()
    if out is None:
        out = torch.zeros_like(x)
    fault = np.array([f.x0, f.y0, f.depth, f.length, f.width, f.strike, f.rake, f.dip, f.slip], dtype=np.float64)
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    L = _lib()
    rc = L.esdg_okada_uplift(int(x.numel()), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                             fault.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(bool(mercator)),
                             int(bool(add)), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s))
    if rc != 0:
        raise RuntimeError(f"esdg_okada_uplift failed ({rc}): {L.esdg_last_error(None).decode()}")
    return out
