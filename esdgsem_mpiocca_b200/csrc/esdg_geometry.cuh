// Curvilinear element geometry on the device: nodal coordinates by the
// transfinite map of an element's boundary curves (bilinear when no side
// is curved), metric terms by the collocation derivative, Jacobian and the
// outward unit normals and scale factors of the four sides -- the host
// set-up's Mesh::element_from_curves / element_geometry (esdg_setup.cpp),
// which restate src/Mesh.cpp:1000-1081, 1619-1650 and 1667-1808, with every
// operation in the same order, so the arrays are the same bits.
//
// Input per element: its 4 corners (x, y) and, per side, a curve flag and
// m + 1 Chebyshev-Gauss-Lobatto samples of the side (x, y), sides 0 bottom,
// 1 right, 2 top, 3 left running from corner ENDS[s][0] to ENDS[s][1], as
// the ISM-V2 reader and the mapped generator store them.  One thread per
// node, NE elements per block; the element's side samples (curved sides as
// given, straight sides sampled from their corners) and its nodal
// coordinates pass through shared memory.
#pragma once

#include <cuda_runtime.h>

namespace esdg {

constexpr int GEO_MAXM = 16;  // highest boundary-curve order

struct GeoConst {
    double xg[16];                // LGL nodes
    double D0[256];               // collocation derivative matrix [ngl][ngl]
    double xc[GEO_MAXM + 1];      // curve samples -cos(k pi / m)
    double wb[GEO_MAXM + 1];      // their barycentric weights
    double tol;                   // sample-coincidence tolerance, 1e-12
    int m;                        // curve order
};

// Curve::eval: the barycentric interpolant of samples f at s (the sample
// itself where s meets a sample point).
__device__ __forceinline__ double geo_eval(const GeoConst& G, const double* f, double s) {
    double num = 0.0, den = 0.0, out = 0.0;
    bool at = false;
    for (int j = 0; j <= G.m; ++j)
        if (fabs(s - G.xc[j]) < G.tol) { at = true; out = f[j]; }
    if (!at) {
        for (int j = 0; j <= G.m; ++j) {
            const double t = G.wb[j] / (s - G.xc[j]);
            num += t * f[j];
            den += t;
        }
        out = num / den;
    }
    return out;
}

__device__ __forceinline__ double geo_transfinite(const GeoConst& G, const double* G1, const double* G2,
                                                  const double* G3, const double* G4, double psi, double eta) {
    const double x1r = geo_eval(G, G1, -1.0), x2r = geo_eval(G, G1, 1.0);
    const double x3r = geo_eval(G, G3, 1.0), x4r = geo_eval(G, G3, -1.0);
    const double x1 = geo_eval(G, G1, psi), x2 = geo_eval(G, G2, eta);
    const double x3 = geo_eval(G, G3, psi), x4 = geo_eval(G, G4, eta);
    return 0.5 * ((1.0 - psi) * x4 + (1.0 + psi) * x2 + (1.0 - eta) * x1 + (1.0 + eta) * x3) -
           0.25 * ((1.0 - psi) * ((1.0 - eta) * x1r + (1.0 + eta) * x4r) +
                   (1.0 + psi) * ((1.0 - eta) * x2r + (1.0 + eta) * x3r));
}

__device__ __forceinline__ double geo_bilinear(const double* c, double psi, double eta) {
    return 0.25 * (c[0] * (1.0 - psi) * (1.0 - eta) + c[1] * (1.0 + psi) * (1.0 - eta) +
                   c[2] * (1.0 + psi) * (1.0 + eta) + c[3] * (1.0 - psi) * (1.0 + eta));
}

struct GeoArgs {
    int K;
    const double* __restrict__ corners;  // [K][4][2]
    const int* __restrict__ curved;      // [K][4]
    const double* __restrict__ curves;   // [K][4][m+1][2]
    double *x, *y, *xXi, *xEta, *yXi, *yEta, *J;  // [K][ngl][ngl]
    double *nxSide, *nySide, *scalSide;           // [K][4][ngl]
};

// elements per block: one thread per node, at most 16 elements (the side
// samples of each stay in shared memory)
template <int NGL>
struct GeoShape {
    static constexpr int N2 = NGL * NGL;
    static constexpr int NE = (256 / N2) > 16 ? 16 : ((256 / N2) > 0 ? (256 / N2) : 1);
    static constexpr int THREADS = NE * N2;
};

template <int NGL>
__global__ void __launch_bounds__(GeoShape<NGL>::THREADS) k_geometry(GeoArgs a, GeoConst G) {
    constexpr int N2 = NGL * NGL, NE = GeoShape<NGL>::NE, MP = GEO_MAXM + 1;
    __shared__ double sG[NE][2][4][MP];  // side samples x, y
    __shared__ double sC[NE][2][4];      // corners x, y
    __shared__ int sCurved[NE];          // any side curved
    __shared__ double sx[NE * N2], sy[NE * N2];
    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    const int e = blockIdx.x * NE + el;
    const bool inb = e < a.K;
    const int m = G.m;
    // corners and side samples of the block's elements
    if (inb && nd < 4) {
        sC[el][0][nd] = a.corners[((long)e * 4 + nd) * 2 + 0];
        sC[el][1][nd] = a.corners[((long)e * 4 + nd) * 2 + 1];
    }
    if (inb && nd == 0) {
        int c = 0;
        for (int s = 0; s < 4; ++s) c |= a.curved[(long)e * 4 + s] ? 1 : 0;
        sCurved[el] = c;
    }
    __syncthreads();
    static constexpr int ends[4][2] = {{0, 1}, {1, 2}, {3, 2}, {0, 3}};
    for (int idx = nd; inb && idx < 4 * (m + 1); idx += N2) {
        const int s = idx / (m + 1), k = idx % (m + 1);
        if (a.curved[(long)e * 4 + s]) {
            const long o = (((long)e * 4 + s) * (m + 1) + k) * 2;
            sG[el][0][s][k] = a.curves[o + 0];
            sG[el][1][s][k] = a.curves[o + 1];
        } else {
            const int p = ends[s][0], q = ends[s][1];
            sG[el][0][s][k] = ((sC[el][0][q] - sC[el][0][p]) * G.xc[k] + sC[el][0][p] + sC[el][0][q]) / 2.0;
            sG[el][1][s][k] = ((sC[el][1][q] - sC[el][1][p]) * G.xc[k] + sC[el][1][p] + sC[el][1][q]) / 2.0;
        }
    }
    __syncthreads();
    const int i = nd % NGL, j = nd / NGL;
    const int s0 = el * N2;
    if (inb) {
        double xp, yp;
        if (sCurved[el]) {
            xp = geo_transfinite(G, sG[el][0][0], sG[el][0][1], sG[el][0][2], sG[el][0][3], G.xg[i], G.xg[j]);
            yp = geo_transfinite(G, sG[el][1][0], sG[el][1][1], sG[el][1][2], sG[el][1][3], G.xg[i], G.xg[j]);
        } else {
            xp = geo_bilinear(sC[el][0], G.xg[i], G.xg[j]);
            yp = geo_bilinear(sC[el][1], G.xg[i], G.xg[j]);
        }
        sx[s0 + nd] = xp;
        sy[s0 + nd] = yp;
    }
    __syncthreads();
    if (!inb) return;
    const long id = (long)e * N2 + nd;
    double A = 0, B = 0, C = 0, Dd = 0;
#pragma unroll
    for (int k = 0; k < NGL; ++k) {
        A += G.D0[i * NGL + k] * sx[s0 + j * NGL + k];
        B += G.D0[j * NGL + k] * sx[s0 + k * NGL + i];
        C += G.D0[i * NGL + k] * sy[s0 + j * NGL + k];
        Dd += G.D0[j * NGL + k] * sy[s0 + k * NGL + i];
    }
    const double Jt = A * Dd - B * C;
    a.x[id] = sx[s0 + nd];
    a.y[id] = sy[s0 + nd];
    a.xXi[id] = A; a.xEta[id] = B; a.yXi[id] = C; a.yEta[id] = Dd; a.J[id] = Jt;
    // side normals: right (i = NGL-1) and left (i = 0) sides from the eta
    // derivatives, bottom (j = 0) and top (j = NGL-1) from the xi ones
    const long so = (long)e * 4 * NGL;
    if (i == NGL - 1) {
        const double sc = sqrt(Dd * Dd + B * B);
        a.scalSide[so + NGL + j] = sc;
        a.nxSide[so + NGL + j] = copysign(1.0, Jt) * (Dd / sc);
        a.nySide[so + NGL + j] = copysign(1.0, Jt) * (-B / sc);
    }
    if (i == 0) {
        const double sc = sqrt(Dd * Dd + B * B);
        a.scalSide[so + 3 * NGL + j] = sc;
        a.nxSide[so + 3 * NGL + j] = -copysign(1.0, Jt) * (Dd / sc);
        a.nySide[so + 3 * NGL + j] = -copysign(1.0, Jt) * (-B / sc);
    }
    if (j == 0) {
        const double sc = sqrt(C * C + A * A);
        a.scalSide[so + i] = sc;
        a.nxSide[so + i] = -copysign(1.0, Jt) * (-C / sc);
        a.nySide[so + i] = -copysign(1.0, Jt) * (A / sc);
    }
    if (j == NGL - 1) {
        const double sc = sqrt(C * C + A * A);
        a.scalSide[so + 2 * NGL + i] = sc;
        a.nxSide[so + 2 * NGL + i] = copysign(1.0, Jt) * (-C / sc);
        a.nySide[so + 2 * NGL + i] = copysign(1.0, Jt) * (A / sc);
    }
}

}  // namespace esdg
