// Sea-surface uplift of a rectangular fault on the device: the vertical
// surface displacement of the Okada (1985) strike-slip and dip-slip
// dislocation, restated from src/okada.cpp:33-249 of the reference (the same
// formulas as the host restatement esdgsem_mpiocca_b200/okada.py, in the
// same order of operations), one thread per node.
//
// Two front-ends: MERCATOR = true is the reference's own geometry (node
// coordinates in kilometres of a Mercator projection of lon/lat, the uplift
// in kilometres inside its lon/lat-aligned box around the epicentre);
// MERCATOR = false is the same dislocation on plane coordinates in metres
// (the synthetic scenarios on a Cartesian square: uplift in metres inside a
// box of half-size 1.5 max(length, width) around the centroid).  The
// fault's scalar terms (angles, their sines and cosines, depth of the lower
// edge, epicentre offsets) are evaluated once on the host.
#pragma once

#include <cuda_runtime.h>

namespace esdg {

struct OkadaConst {
    double x0, y0;               // centroid (m) or epicentre lon/lat (deg)
    double halfl, width, hh;     // half length, width, depth of the lower edge
    double sn_l, cs_l;           // sin / cos of the dip
    double sn_t, cs_t;           // sin / cos of the strike
    double del_x, del_y;         // epicentre offset of the reference
    double ds, dd;               // strike-slip and dip-slip dislocations
    double reach;                // Cartesian: box half-size
    // Mercator: the box and the reference's lon/lat origin
    double R, rad, xlower, xupper, ylower, yupper, xo, yo, yl, xl0;
};

__device__ __forceinline__ double okada_strike_slip(const OkadaConst& c, double x2, double y1, double y2) {
    // src/okada.cpp:196-222
    const double sn = c.sn_l, cs = c.cs_l;
    const double q = x2 * sn - c.hh * cs;
    const double d_bar = y2 * sn - q * cs;
    const double r = sqrt(y1 * y1 + y2 * y2 + q * q);
    const double a4 = 0.5 * 1.0 / cs * (log(r + d_bar) - sn * log(r + y2));
    return -(d_bar * q / r / (r + y2) + q * sn / (r + y2) + a4 * sn) / (2.0 * M_PI);
}

__device__ __forceinline__ double okada_dip_slip(const OkadaConst& c, double x2, double y1, double y2) {
    // src/okada.cpp:224-249
    const double sn = c.sn_l, cs = c.cs_l;
    const double q = x2 * sn - c.hh * cs;
    const double d_bar = y2 * sn - q * cs;
    const double r = sqrt(y1 * y1 + y2 * y2 + q * q);
    const double xx = sqrt(y1 * y1 + q * q);
    const double a5 = 0.5 * 2 / cs * atan((y2 * (xx + q * cs) + xx * (r + xx) * sn) / y1 / (r + xx) / cs);
    return -(d_bar * q / r / (r + y1) + sn * atan(y1 * y2 / q / r) - a5 * sn * cs) / (2.0 * M_PI);
}

// Vertical displacement from the four corners (src/okada.cpp:160-181).
__device__ __forceinline__ double okada_dislocation(const OkadaConst& c, double x1, double x2) {
    const double p = x2 * c.cs_l + c.hh * c.sn_l;
    const double f1 = okada_strike_slip(c, x2, x1 + c.halfl, p);
    const double f2 = okada_strike_slip(c, x2, x1 + c.halfl, p - c.width);
    const double f3 = okada_strike_slip(c, x2, x1 - c.halfl, p);
    const double f4 = okada_strike_slip(c, x2, x1 - c.halfl, p - c.width);
    const double g1 = okada_dip_slip(c, x2, x1 + c.halfl, p);
    const double g2 = okada_dip_slip(c, x2, x1 + c.halfl, p - c.width);
    const double g3 = okada_dip_slip(c, x2, x1 - c.halfl, p);
    const double g4 = okada_dip_slip(c, x2, x1 - c.halfl, p - c.width);
    return (f1 - f2 - f3 + f4) * c.ds + (g1 - g2 - g3 + g4) * c.dd;
}

// out[i] (ADD: out[i] +) the uplift at node i.
template <bool MERCATOR>
__global__ void k_okada(long n, const double* __restrict__ x, const double* __restrict__ y, OkadaConst c,
                        double* __restrict__ out, int add) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double u = 0.0;
    if (!MERCATOR) {
        const double xi = x[i], yi = y[i];
        if (fabs(xi - c.x0) <= c.reach && fabs(yi - c.y0) <= c.reach) {
            const double dx = (xi - c.x0) - c.del_x;
            const double dy = (yi - c.y0) + c.del_y;
            const double x1 = dx * c.sn_t + dy * c.cs_t;
            const double x2 = -(dx * c.cs_t - dy * c.sn_t);
            u = okada_dislocation(c, x1, x2);
            if (!isfinite(u)) u = 0.0;
        }
    } else {
        // src/okada.cpp:33-195: nodes in Mercator kilometres, uplift in kilometres
        const double xloc = x[i] * 1000.0, yloc = y[i] * 1000.0;
        if (xloc >= c.xlower && xloc <= c.xupper && yloc >= c.ylower && yloc <= c.yupper) {
            const double xd = (xloc / c.R) * (180.0 / M_PI);
            const double yd = atan(sinh(yloc / c.R)) * (180.0 / M_PI);
            const double xl = c.R * cos(c.rad * yd) * (c.x0 - c.xo) * c.rad + c.del_x;
            const double yy = c.R * (yd - c.yo) * c.rad;
            const double xx = c.R * cos(c.rad * yd) * (xd - c.xo) * c.rad;
            const double x1 = (xx - xl) * c.sn_t + (yy - c.yl) * c.cs_t;
            const double x2 = -((xx - xl) * c.cs_t - (yy - c.yl) * c.sn_t);
            u = okada_dislocation(c, x1, x2) / 1000.0;
        }
    }
    out[i] = add ? out[i] + u : u;
}

}  // namespace esdg
