// Device-side point physics of the ES-DGSEM shallow-water scheme: the
// entropy-conservative two-point volume fluxes and the entropy-stable
// interface fluxes.  Expressions keep the association order of the reference
// kernels they restate, so that results match the reference to round-off.
#pragma once

#include <cuda_runtime.h>

namespace esdg {

struct PhysConst {
    double g, half_g, fourth_g, geomFace, PosPresTOL;
    double eps0, sigmaMin, sigmaMax, ZeroTOL;
    // energy ratio below which log10(ratio) < sigmaMin holds with margin
    // (10^sigmaMin (1 - 1e-12)): the sensor returns 0 without log10/sin
    double sensor_skip;
    int ES;
};

// Two-point fluxes F#, G# of okl/DG/VolumeKernelFluxDiffV99.okl:17-57 for
// the pair (L, R), contracted with the averaged metric terms (a, b):
//   xi  direction: a = Y_eta, b = X_eta, F = a*f - b*g
//   eta direction: a = Y_xi,  b = X_xi,  G = -a*f + b*g
__device__ __forceinline__ void two_point_xi(double fourth_g, double half_g, double hL, double huL, double hvL,
                                             double iL, double hR, double huR, double hvR, double iR, double aL,
                                             double aR, double bL, double bR, double& F1, double& F2,
                                             double& F3) {
    const double h_A = fourth_g * (hL + hR) * (hL + hR);
    const double h2_A = 0.5 * (hL * hL + hR * hR);
    const double hu_A = 0.5 * (huL + huR);
    const double hv_A = 0.5 * (hvL + hvR);
    const double u_A = 0.5 * (huL * iL + huR * iR);
    const double v_A = 0.5 * (hvL * iL + hvR * iR);
    const double a = 0.5 * (aL + aR);
    const double b = 0.5 * (bL + bR);
    const double p = h_A - half_g * h2_A;
    F1 = a * hu_A - b * hv_A;
    F2 = a * (hu_A * u_A + p) - b * hv_A * u_A;
    F3 = a * (hu_A * v_A) - b * (hv_A * v_A + p);
}

__device__ __forceinline__ void two_point_eta(double fourth_g, double half_g, double hL, double huL, double hvL,
                                              double iL, double hR, double huR, double hvR, double iR, double aL,
                                              double aR, double bL, double bR, double& G1, double& G2,
                                              double& G3) {
    const double h_A = fourth_g * (hL + hR) * (hL + hR);
    const double h2_A = 0.5 * (hL * hL + hR * hR);
    const double hu_A = 0.5 * (huL + huR);
    const double hv_A = 0.5 * (hvL + hvR);
    const double u_A = 0.5 * (huL * iL + huR * iR);
    const double v_A = 0.5 * (hvL * iL + hvR * iR);
    const double a = 0.5 * (aL + aR);
    const double b = 0.5 * (bL + bR);
    const double p = h_A - half_g * h2_A;
    G1 = -a * hu_A + b * hv_A;
    G2 = -a * (hu_A * u_A + p) + b * hv_A * u_A;
    G3 = -a * (hu_A * v_A) + b * (hv_A * v_A + p);
}

// Entropy-stable interface flux at one face node, L = master side state,
// R = slave side state in the master's node order, n = master's outward unit
// normal.  NUMFLUX 0: okl/RiemannSolvers/calcESFlux.okl:17-215;
// 3: okl/RiemannSolvers/calcESFluxRotated.okl:17-214; 2: the Rusanov-type
// ES flux of okl/RiemannSolvers/calcLFTypeESFlux.okl:17-195 with the right
// state reversed like the other two (the reference call site of that kernel
// passes one argument too many, src/deviceclass.cpp:1004).
template <int NUMFLUX>
__device__ __forceinline__ void es_flux(const PhysConst& c, double nx, double ny, double hL, double huL,
                                        double hvL, double hR, double huR, double hvR, double bL, double bR,
                                        double& N0, double& N1, double& N2) {
    const double tol = c.PosPresTOL, g = c.g;
    double uL, vL, uR, vR;
    if (NUMFLUX == 0) {
        if (hL >= tol) { uL = huL / hL; vL = hvL / hL; } else { hL = 0.0; uL = 0.0; vL = 0.0; }
        if (hR >= tol) { uR = huR / hR; vR = hvR / hR; } else { hR = 0.0; uR = 0.0; vR = 0.0; }
        const double avgH = 0.5 * (hL + hR), avgH2 = 0.5 * (hL * hL + hR * hR);
        const double avgU = 0.5 * (uL + uR), avgV = 0.5 * (vL + vR);
        const double normV = avgU * nx + avgV * ny;
        N0 = avgH * normV;
        N1 = avgH * avgU * normV + (0.5 * g * avgH2) * nx;
        N2 = avgH * avgV * normV + (0.5 * g * avgH2) * ny;
        if (c.ES) {
            const double cL = g * hL, cR = g * hR;
            const double avgC = sqrt(fabs(0.5 * (cL + cR)));
            const double q1L = g * (hL + bL) - 0.5 * uL * uL - 0.5 * vL * vL;
            const double q1R = g * (hR + bR) - 0.5 * uR * uR - 0.5 * vR * vR;
            const double j1 = q1R - q1L, j2 = uR - uL, j3 = vR - vL;
            const double R21 = avgU + nx * avgC, R22 = ny, R23 = avgU - nx * avgC;
            const double R31 = avgV + ny * avgC, R32 = nx, R33 = avgV - ny * avgC;
            const double SL11 = 0.5 / g * fabs(nx * avgU + ny * avgV + avgC);
            const double SL22 = fabs(avgH * (nx * avgU + ny * avgV));
            const double SL33 = 0.5 / g * fabs(nx * avgU + ny * avgV - avgC);
            const double RSL11 = 1.0 * SL11, RSL12 = 0.0, RSL13 = 1.0 * SL33;
            const double RSL21 = R21 * SL11, RSL22 = R22 * SL22, RSL23 = R23 * SL33;
            const double RSL31 = R31 * SL11, RSL32 = R32 * SL22, RSL33 = R33 * SL33;
            const double M11 = RSL11 * 1.0 + RSL12 * 0.0 + RSL13 * 1.0;
            const double M12 = RSL11 * R21 + RSL12 * R22 + RSL13 * R23;
            const double M13 = RSL11 * R31 + RSL12 * R32 + RSL13 * R33;
            const double M21 = RSL21 * 1.0 + RSL22 * 0.0 + RSL23 * 1.0;
            const double M22 = RSL21 * R21 + RSL22 * R22 + RSL23 * R23;
            const double M23 = RSL21 * R31 + RSL22 * R32 + RSL23 * R33;
            const double M31 = RSL31 * 1.0 + RSL32 * 0.0 + RSL33 * 1.0;
            const double M32 = RSL31 * R21 + RSL32 * R22 + RSL33 * R23;
            const double M33 = RSL31 * R31 + RSL32 * R32 + RSL33 * R33;
            N0 += -0.5 * (M11 * j1 + M12 * j2 + M13 * j3);
            N1 += -0.5 * (M21 * j1 + M22 * j2 + M23 * j3);
            N2 += -0.5 * (M31 * j1 + M32 * j2 + M33 * j3);
        }
    } else if (NUMFLUX == 3) {
        if (hL > tol) { uL = huL / hL; vL = hvL / hL; } else { uL = 0.0; vL = 0.0; }
        if (hR > tol) { uR = huR / hR; vR = hvR / hR; } else { uR = 0.0; vR = 0.0; }
        const double vLn = nx * uL + ny * vL, vLt = -ny * uL + nx * vL;
        const double vRn = nx * uR + ny * vR, vRt = -ny * uR + nx * vR;
        const double avgH = 0.5 * (hL + hR), avgH2 = 0.5 * (hL * hL + hR * hR);
        const double avgU = 0.5 * (vLn + vRn), avgV = 0.5 * (vLt + vRt);
        double A0 = avgH * avgU;
        double A1 = avgH * avgU * avgU + (0.5 * g * avgH2);
        double A2 = avgH * avgV * avgU;
        if (c.ES) {
            const double cL = g * hL, cR = g * hR;
            const double avgC = sqrt(fabs(0.5 * (cL + cR)));
            const double q1L = g * (hL + bL) - 0.5 * vLn * vLn - 0.5 * vLt * vLt;
            const double q1R = g * (hR + bR) - 0.5 * vRn * vRn - 0.5 * vRt * vRt;
            const double j1 = q1R - q1L, j2 = vRn - vLn, j3 = vRt - vLt;
            const double R21 = avgU + avgC, R22 = 0.0, R23 = avgU - avgC;
            const double R31 = avgV, R32 = 1.0, R33 = avgV;
            const double SL11 = 0.5 / g * fabs(avgU + avgC);
            const double SL22 = fabs(avgH * avgU);
            const double SL33 = 0.5 / g * fabs(avgU - avgC);
            const double RSL11 = 1.0 * SL11, RSL12 = 0.0, RSL13 = 1.0 * SL33;
            const double RSL21 = R21 * SL11, RSL22 = R22 * SL22, RSL23 = R23 * SL33;
            const double RSL31 = R31 * SL11, RSL32 = R32 * SL22, RSL33 = R33 * SL33;
            const double M11 = RSL11 * 1.0 + RSL12 * 0.0 + RSL13 * 1.0;
            const double M12 = RSL11 * R21 + RSL12 * R22 + RSL13 * R23;
            const double M13 = RSL11 * R31 + RSL12 * R32 + RSL13 * R33;
            const double M21 = RSL21 * 1.0 + RSL22 * 0.0 + RSL23 * 1.0;
            const double M22 = RSL21 * R21 + RSL22 * R22 + RSL23 * R23;
            const double M23 = RSL21 * R31 + RSL22 * R32 + RSL23 * R33;
            const double M31 = RSL31 * 1.0 + RSL32 * 0.0 + RSL33 * 1.0;
            const double M32 = RSL31 * R21 + RSL32 * R22 + RSL33 * R23;
            const double M33 = RSL31 * R31 + RSL32 * R32 + RSL33 * R33;
            A0 += -0.5 * (M11 * j1 + M12 * j2 + M13 * j3);
            A1 += -0.5 * (M21 * j1 + M22 * j2 + M23 * j3);
            A2 += -0.5 * (M31 * j1 + M32 * j2 + M33 * j3);
        }
        N0 = A0;
        N1 = nx * A1 - ny * A2;
        N2 = ny * A1 + nx * A2;
    } else {
        if (hL > tol) { uL = huL / hL; vL = hvL / hL; } else { uL = 0.0; vL = 0.0; }
        if (hR > tol) { uR = huR / hR; vR = hvR / hR; } else { uR = 0.0; vR = 0.0; }
        const double avgH = 0.5 * (hL + hR), avgH2 = 0.5 * (hL * hL + hR * hR);
        const double avgU = 0.5 * (uL + uR), avgV = 0.5 * (vL + vR);
        const double normV = avgU * nx + avgV * ny;
        N0 = avgH * normV;
        N1 = avgH * avgU * normV + (0.5 * g * avgH2) * nx;
        N2 = avgH * avgV * normV + (0.5 * g * avgH2) * ny;
        if (c.ES) {
            const double cL = (hL > tol) ? sqrt(g * hL) : 0.0;
            const double cR = (hR > tol) ? sqrt(g * hR) : 0.0;
            const double q1L = g * (hL + bL) - 0.5 * uL * uL - 0.5 * vL * vL;
            const double q1R = g * (hR + bR) - 0.5 * uR * uR - 0.5 * vR * vR;
            const double j1 = q1R - q1L, j2 = uR - uL, j3 = vR - vL;
            const double H12 = avgU, H13 = avgV;
            const double H21 = avgU, H22 = g * avgH + avgU * avgU, H23 = avgU * avgV;
            const double H31 = avgV, H32 = avgU * avgV, H33 = g * avgH + avgV * avgV;
            const double lL = cL + fmax(fabs(uL), fabs(vL));
            const double lR = cR + fmax(fabs(uR), fabs(vR));
            const double lam = fmax(lL, lR) / g;
            N0 += -0.5 * lam * (1.0 * j1 + H12 * j2 + H13 * j3);
            N1 += -0.5 * lam * (H21 * j1 + H22 * j2 + H23 * j3);
            N2 += -0.5 * lam * (H31 * j1 + H32 * j2 + H33 * j3);
        }
    }
}

// Solid-wall ghost state (okl/GatherEdgeData/SolidWalls.okl:150-173): same
// depth, normal momentum reflected.
__device__ __forceinline__ void wall_ghost(double nx, double ny, double h, double hu, double hv, double& gh,
                                           double& ghu, double& ghv) {
    const double v_n = nx * hu + ny * hv;
    const double v_t = -ny * hu + nx * hv;
    gh = h;
    ghu = -nx * v_n - ny * v_t;
    ghv = -ny * v_n + nx * v_t;
}

// Offset of trace node i of side s inside one element's [ngl][ngl] block
// (sides 0 bottom, 1 right, 2 top, 3 left; okl/GatherEdgeData/SolidWalls.okl:74-89).
__device__ __forceinline__ int trace_offset(int side, int i, int ngl) {
    switch (side) {
        case 0: return i;
        case 2: return ngl * ngl - ngl + i;
        case 3: return i * ngl;
        default: return (i + 1) * ngl - 1;
    }
}

// Testcase 1 (manufactured solution on a Cartesian mesh with Dirichlet
// boundaries): H = 8 + cos x sin y cos t, u = 1/2, v = 3/2, h = H - b.
// The exact state (okl/GatherEdgeData/Dirichlet_ConvTest.okl:14-26), used as
// the outer state of boundary faces at the stage time.
__device__ __forceinline__ void conv_exact(double x, double y, double t, double b, double& q1, double& q2,
                                           double& q3) {
    q1 = (8.0 + cos(x) * sin(y) * cos(t) - b);
    q2 = 0.5 * (8.0 + cos(x) * sin(y) * cos(t) - b);
    q3 = 1.5 * (8.0 + cos(x) * sin(y) * cos(t) - b);
}

// Its source term (okl/ManufacturedSolutions/S_ConvTest.okl), added to the
// right-hand side after the volume and surface terms, before the update.
__device__ __forceinline__ void conv_source(double g, double x, double y, double t, double Bx, double By, double B,
                                            double& s0, double& s1, double& s2) {
    const double sinY = sin(y), sinX = sin(x), cosY = cos(y), cosX = cos(x);
    const double H = 8.0 + cosX * sinY * cos(t);
    const double Ht = -cosX * sinY * sin(t);
    const double Hx = -sinX * sinY * cos(t);
    const double Hy = cosX * cosY * cos(t);
    const double u = 0.5, v = 1.5;
    s0 = Ht + u * (Hx - Bx) + v * (Hy - By);
    s1 = u * Ht + u * u * (Hx - Bx) + u * v * (Hy - By) + g * Hx * (H - B);
    s2 = v * Ht + u * v * (Hx - Bx) + v * v * (Hy - By) + g * Hy * (H - B);
}

// Order-preserving map of non-negative doubles to unsigned 64-bit keys for
// atomicMax (NaN maps above +inf, so a NaN anywhere shows up in the max).
__device__ __forceinline__ unsigned long long dbl_key(double v) {
    if (isnan(v)) return ~0ull;
    const long long b = __double_as_longlong(v);
    return (b < 0) ? 0ull : (unsigned long long)b;
}

}  // namespace esdg
