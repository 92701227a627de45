// Partial-dry treatment (PartialDryTreatment = 1): on elements with a node
// below PosPresTOL the momentum part of the volume term is replaced by a
// finite-difference form that keeps the hydrostatic balance at wet/dry
// fronts.  okl/PartialDryTreatment/FindDryElements.okl:16-63 (the flag)
// and okl/PartialDryTreatment/VolumeKernelFD.okl:33-343 (the replacement),
// called by the reference right after the volume kernel and before the
// surface lift (src/deviceclass.cpp:987-991), so the surface terms are added
// on top as usual.
#pragma once

#include "esdg_physics.cuh"

namespace esdg {

// dry[e] = 1 when min(1, h over the element's nodes) < PosPresTOL (fmin
// ignores NaN, as in the reference).  One thread per element.
template <int NGL>
__global__ void k_find_dry(int K, const double* __restrict__ q, int* __restrict__ dry, double tol) {
    constexpr int N2 = NGL * NGL;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= K) return;
    const double* h = q + (long)e * 3 * N2;
    double m = 1.0;
#pragma unroll
    for (int k = 0; k < N2; ++k) m = fmin(h[k], m);
    dry[e] = (m < tol) ? 1 : 0;
}

// The momentum volume terms (r1, r2) of node (i = eta, j = xi) of a
// partly dry element.  hel: the element's h [N2] (xi fastest), bel: its b
// [N2]; Dc, Dup, Ddn: central, forward ("upwind") and backward
// ("downwind") difference matrices [N2].  F = G = g h and the boundary
// terms g/2 h^2 as in the reference; each difference uses a neighbour only
// where that neighbour is wet, the same operand order throughout.
template <int NGL>
__device__ __forceinline__ void pd_volume(const PhysConst& c, const double* __restrict__ Dc,
                                          const double* __restrict__ Dup, const double* __restrict__ Ddn,
                                          const double* hel, const double* __restrict__ bel, int i, int j, double Ye,
                                          double Yx, double Xe, double Xx, double J, double& r1, double& r2) {
    const double tol = c.PosPresTOL, g = c.g;
    const double h = hel[i * NGL + j], b = bel[i * NGL + j];
    const double hxm = j > 0 ? hel[i * NGL + j - 1] : 0.0;
    const double hxp = j < NGL - 1 ? hel[i * NGL + j + 1] : 0.0;
    const double hym = i > 0 ? hel[(i - 1) * NGL + j] : 0.0;
    const double hyp = i < NGL - 1 ? hel[(i + 1) * NGL + j] : 0.0;
    // F2_2 = G3_2 = g h at a node
    auto gh = [&](int ii, int jj) { return g * hel[ii * NGL + jj]; };
    double Fxi = 0.0, Feta = 0.0, Bxi = 0.0, Beta = 0.0;
    if (h > tol) {
        // xi: along the row, neighbours (i, j -+ 1)
        if (j == 0) {
            if (hxp > tol) {
                const double dp = Dup[j * NGL + 1], d0 = Dup[j * NGL + 0];
                Fxi = d0 * gh(i, j) + dp * gh(i, j + 1);
                Bxi = d0 * b + dp * bel[i * NGL + j + 1];
            }
        }
        if (j == NGL - 1) {
            if (hxm > tol) {
                const double d0 = Ddn[j * NGL + NGL - 1], dm = Ddn[j * NGL + NGL - 2];
                Fxi = dm * gh(i, j - 1) + d0 * gh(i, j);
                Bxi = dm * bel[i * NGL + j - 1] + d0 * b;
            }
        }
        if (j > 0 && j < NGL - 1) {
            if (hxp > tol) {
                if (hxm > tol) {
                    const double dp = Dc[j * NGL + j + 1], dm = Dc[j * NGL + j - 1];
                    Fxi = dm * gh(i, j - 1) + dp * gh(i, j + 1);
                    Bxi = dm * bel[i * NGL + j - 1] + dp * bel[i * NGL + j + 1];
                } else {
                    const double dp = Dup[j * NGL + j + 1], d0 = Dup[j * NGL + j];
                    Fxi = d0 * gh(i, j) + dp * gh(i, j + 1);
                    Bxi = d0 * b + dp * bel[i * NGL + j + 1];
                }
            } else if (hxm > tol) {
                const double d0 = Ddn[j * NGL + j], dm = Ddn[j * NGL + j - 1];
                Fxi = dm * gh(i, j - 1) + d0 * gh(i, j);
                Bxi = dm * bel[i * NGL + j - 1] + d0 * b;
            }
        }
        // eta: along the column, neighbours (i -+ 1, j)
        if (i == 0) {
            if (hyp > tol) {
                const double dp = Dup[i * NGL + 1], d0 = Dup[i * NGL + 0];
                Feta = d0 * gh(i, j) + dp * gh(i + 1, j);
                Beta = d0 * b + dp * bel[(i + 1) * NGL + j];
            }
        }
        if (i == NGL - 1) {
            if (hym > tol) {
                const double d0 = Ddn[i * NGL + NGL - 1], dm = Ddn[i * NGL + NGL - 2];
                Feta = dm * gh(i - 1, j) + d0 * gh(i, j);
                Beta = dm * bel[(i - 1) * NGL + j] + d0 * b;
            }
        }
        if (i > 0 && i < NGL - 1) {
            if (hyp > tol) {
                if (hym > tol) {
                    const double dp = Dc[i * NGL + i + 1], dm = Dc[i * NGL + i - 1];
                    Feta = dm * gh(i - 1, j) + dp * gh(i + 1, j);
                    Beta = dm * bel[(i - 1) * NGL + j] + dp * bel[(i + 1) * NGL + j];
                } else {
                    const double dp = Dup[i * NGL + i + 1], d0 = Dup[i * NGL + i];
                    Feta = d0 * gh(i, j) + dp * gh(i + 1, j);
                    Beta = d0 * b + dp * bel[(i + 1) * NGL + j];
                }
            } else if (hym > tol) {
                const double d0 = Ddn[i * NGL + i], dm = Ddn[i * NGL + i - 1];
                Feta = dm * gh(i - 1, j) + d0 * gh(i, j);
                Beta = dm * bel[(i - 1) * NGL + j] + d0 * b;
            }
        }
    }
    // boundary terms g/2 h^2 at the element's edges (F and G alike)
    const double bd = c.half_g * h * h;
    double Fxib = 0.0, Fetab = 0.0;
    if (j == 0) Fxib += c.geomFace * bd;
    if (j == NGL - 1) Fxib += -c.geomFace * bd;
    if (i == 0) Fetab += c.geomFace * bd;
    if (i == NGL - 1) Fetab += -c.geomFace * bd;
    const double fx2 = Ye * Fxib - Yx * Fetab;
    const double fx2_2 = h * (Ye * Fxi - Yx * Feta);
    const double gy3 = -Xe * Fxib + Xx * Fetab;
    const double gy3_2 = h * (-Xe * Fxi + Xx * Feta);
    const double bx = Ye * Bxi - Yx * Beta;
    const double by = -Xe * Bxi + Xx * Beta;
    const double d2 = fx2_2 + fx2;
    const double d3 = gy3_2 + gy3;
    r1 = -J * d2 - g * J * h * bx;
    r2 = -J * d3 - g * J * h * by;
}

}  // namespace esdg
