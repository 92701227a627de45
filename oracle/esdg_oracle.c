/*
 * ORACLE -- test infrastructure only.
 *
 * Plain-C, single-threaded (optionally OpenMP over elements/faces) restatement
 * of the ESDGSEM_MPIOCCA per-step kernels and of deviceclass::DGtimeloop.
 * It is what the CUDA engine's results are compared with; nothing in the
 * engine links or calls it.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it.
 *
 * Every routine cites the reference file:line it restates (paths relative to
 * the ESDGSEM_MPIOCCA tree).  Arithmetic is written in the same association
 * order as the reference so that the two agree to the last bit when built
 * without FMA contraction (-ffp-contract=off).
 *
 * Layouts: q/Qt/gRK [K][3][ngl][ngl] (xi fastest), geometry [K][ngl][ngl],
 * face traces [F][3][ngl], face geometry [F][ngl], EdgeData [F][8],
 * ElemToEdge (1-based) / ElemEdgeMasterSlave / ElemEdgeOrientation [K][4].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NEQ 3

typedef struct {
    int ngl;
    double g_const, half_g, fourth_g, geomFace, PosPresTOL;
    double eps0, sigmaMin, sigmaMax, ZeroTOL, PI;
    int ES;
} oconst;

static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }

static void fill_const(oconst* c, int ngl, double g, double geomFace, double PosPresTOL, int ES, double eps0,
                       double sigmaMin, double sigmaMax) {
    /* src/deviceclass.cpp:131-205 (JIT constants) */
    c->ngl = ngl;
    c->g_const = g;
    c->half_g = 0.5 * g;
    c->fourth_g = 0.25 * g;
    c->geomFace = geomFace;
    c->PosPresTOL = PosPresTOL;
    c->ES = ES;
    c->eps0 = eps0;
    c->sigmaMin = sigmaMin;
    c->sigmaMax = sigmaMax;
    c->ZeroTOL = pow(10.0, -5);
    c->PI = M_PI;
}

/* --- okl/GatherEdgeData/CollectEdgeData_Bottom.okl:16-134 ------------------ */
void oracle_collect_bottom(int F, int ngl, const int* EdgeData, const double* B, double* bL, double* bR) {
    const int n2 = ngl * ngl;
    for (int ifa = 0; ifa < F; ++ifa)
        for (int i = 0; i < ngl; ++i) {
            const int iel = EdgeData[8 * ifa], ier = EdgeData[8 * ifa + 1];
            const int isl = EdgeData[8 * ifa + 2], isr = EdgeData[8 * ifa + 3];
            const int cpuL = EdgeData[8 * ifa + 5], cpuR = EdgeData[8 * ifa + 6];
            const long x = (long)ifa * ngl + i;
            bL[x] = 0.0;
            bR[x] = 0.0;
            long idL = 0, idR = 0;
            if (cpuL == 0) {
                switch (isl) {
                    case 0: idL = (long)iel * n2 + i; break;
                    case 2: idL = (long)iel * n2 + n2 - ngl + i; break;
                    case 3: idL = (long)iel * n2 + i * ngl; break;
                    case 1: idL = (long)iel * n2 + (i + 1) * ngl - 1; break;
                }
                bL[x] = B[idL];
            }
            if (cpuR == 0) {
                switch (isr) {
                    case 0: idR = (long)ier * n2 + i; break;
                    case 2: idR = (long)ier * n2 + n2 - ngl + i; break;
                    case 3: idR = (long)ier * n2 + i * ngl; break;
                    case 1: idR = (long)ier * n2 + (i + 1) * ngl - 1; break;
                }
                bR[x] = B[idR];
            }
            if (cpuL == -1) bL[x] = bR[x];
            if (cpuR == -1) bR[x] = bL[x];
        }
}

static inline long trace_index(int e, int side, int i, int ngl, int neq) {
    const long n2 = (long)ngl * ngl;
    switch (side) {
        case 0: return (long)e * n2 * neq + i;
        case 2: return (long)e * n2 * neq + n2 - ngl + i;
        case 3: return (long)e * n2 * neq + (long)i * ngl;
        default: return (long)e * n2 * neq + (long)(i + 1) * ngl - 1;
    }
}

/* --- okl/GatherEdgeData/SolidWalls.okl:16-207 ------------------------------ */
void oracle_collect_edge_walls(int F, int ngl, const int* EdgeData, const double* Q, const double* nxa,
                               const double* nya, double* qL, double* qR) {
    const int n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int ifa = 0; ifa < F; ++ifa)
        for (int i = 0; i < ngl; ++i) {
            const int iel = EdgeData[8 * ifa], ier = EdgeData[8 * ifa + 1];
            const int isl = EdgeData[8 * ifa + 2], isr = EdgeData[8 * ifa + 3];
            const int cpuL = EdgeData[8 * ifa + 5], cpuR = EdgeData[8 * ifa + 6];
            const long eid = (long)ifa * ngl * NEQ + i, ex = (long)ifa * ngl + i;
            const double nx = nxa[ex], ny = nya[ex];
            double L[3] = {0, 0, 0}, R[3] = {0, 0, 0};
            if (cpuL == 0) {
                const long id = trace_index(iel, isl, i, ngl, NEQ);
                L[0] = Q[id]; L[1] = Q[id + n2]; L[2] = Q[id + 2 * n2];
            }
            if (cpuR == 0) {
                const long id = trace_index(ier, isr, i, ngl, NEQ);
                R[0] = Q[id]; R[1] = Q[id + n2]; R[2] = Q[id + 2 * n2];
            }
            if (cpuL == -1) {
                const double vx = R[1], vy = R[2];
                const double v_n = nx * vx + ny * vy, v_t = -ny * vx + nx * vy;
                L[0] = R[0];
                L[1] = -nx * v_n - ny * v_t;
                L[2] = -ny * v_n + nx * v_t;
            }
            if (cpuR == -1) {
                const double vx = L[1], vy = L[2];
                const double v_n = nx * vx + ny * vy, v_t = -ny * vx + nx * vy;
                R[0] = L[0];
                R[1] = -nx * v_n - ny * v_t;
                R[2] = -ny * v_n + nx * v_t;
            }
            qL[eid] = L[0]; qL[eid + ngl] = L[1]; qL[eid + 2 * ngl] = L[2];
            qR[eid] = R[0]; qR[eid + ngl] = R[1]; qR[eid + 2 * ngl] = R[2];
        }
}

/* --- Testcase 1: okl/GatherEdgeData/Dirichlet_ConvTest.okl:14-185, the exact
 * state H = 8 + cos x sin y cos t (minus b), u = 1/2, v = 3/2 outside the
 * boundary faces at the stage time t. */
static void conv_qnodal(double x, double y, double t, double b, double* q) {
    q[0] = (8.0 + cos(x) * sin(y) * cos(t) - b);
    q[1] = 0.5 * (8.0 + cos(x) * sin(y) * cos(t) - b);
    q[2] = 1.5 * (8.0 + cos(x) * sin(y) * cos(t) - b);
}

static void collect_edge_conv(int F, int ngl, const int* EdgeData, const double* Q, const double* X, const double* Y,
                              const double* bL, const double* bR, double t, double* qL, double* qR) {
    const int n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int ifa = 0; ifa < F; ++ifa)
        for (int i = 0; i < ngl; ++i) {
            const int iel = EdgeData[8 * ifa], ier = EdgeData[8 * ifa + 1];
            const int isl = EdgeData[8 * ifa + 2], isr = EdgeData[8 * ifa + 3];
            const int cpuL = EdgeData[8 * ifa + 5], cpuR = EdgeData[8 * ifa + 6];
            const long eid = (long)ifa * ngl * NEQ + i, ex = (long)ifa * ngl + i;
            double L[3] = {0, 0, 0}, R[3] = {0, 0, 0};
            long xl = 0, xr = 0;
            if (cpuL == 0) {
                const long id = trace_index(iel, isl, i, ngl, NEQ);
                xl = trace_index(iel, isl, i, ngl, 1);
                L[0] = Q[id]; L[1] = Q[id + n2]; L[2] = Q[id + 2 * n2];
            }
            if (cpuR == 0) {
                const long id = trace_index(ier, isr, i, ngl, NEQ);
                xr = trace_index(ier, isr, i, ngl, 1);
                R[0] = Q[id]; R[1] = Q[id + n2]; R[2] = Q[id + 2 * n2];
            }
            if (cpuL == -1) conv_qnodal(X[xr], Y[xr], t, bR[ex], L);
            if (cpuR == -1) conv_qnodal(X[xl], Y[xl], t, bL[ex], R);
            qL[eid] = L[0]; qL[eid + ngl] = L[1]; qL[eid + 2 * ngl] = L[2];
            qR[eid] = R[0]; qR[eid + ngl] = R[1]; qR[eid + 2 * ngl] = R[2];
        }
}

/* --- Testcase 1: okl/ManufacturedSolutions/S_ConvTest.okl (addS) ----------- */
static void add_conv_source(const oconst* c, int K, const double* Bx, const double* By, const double* B,
                            const double* X, const double* Y, double t, double* Qt) {
    const int ngl = c->ngl, n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e)
        for (int k = 0; k < n2; ++k) {
            const long x = (long)e * n2 + k, id = (long)e * n2 * NEQ + k;
            const double sinY = sin(Y[x]), sinX = sin(X[x]), cosY = cos(Y[x]), cosX = cos(X[x]);
            const double H = 8.0 + cosX * sinY * cos(t);
            const double Ht = -cosX * sinY * sin(t);
            const double Hx = -sinX * sinY * cos(t);
            const double Hy = cosX * cosY * cos(t);
            const double u = 0.5, v = 1.5;
            Qt[id] += Ht + u * (Hx - Bx[x]) + v * (Hy - By[x]);
            Qt[id + n2] += u * Ht + u * u * (Hx - Bx[x]) + u * v * (Hy - By[x]) + c->g_const * Hx * (H - B[x]);
            Qt[id + 2 * n2] += v * Ht + u * v * (Hx - Bx[x]) + v * v * (Hy - By[x]) + c->g_const * Hy * (H - B[x]);
        }
}

/* --- okl/DG/VolumeKernelFluxDiffV99.okl:17-57 two-point fluxes ------------- */
static inline void Fvol(const oconst* c, double q1L, double q2L, double q3L, double qInvL, double q1R, double q2R,
                        double q3R, double qInvR, double YetaL, double YetaR, double XetaL, double XetaR, double* F1,
                        double* F2, double* F3) {
    const double h_A = c->fourth_g * (q1L + q1R) * (q1L + q1R);
    const double h2_A = 0.5 * (q1L * q1L + q1R * q1R);
    const double hu_A = 0.5 * (q2L + q2R);
    const double hv_A = 0.5 * (q3L + q3R);
    const double u_A = 0.5 * (q2L * qInvL + q2R * qInvR);
    const double v_A = 0.5 * (q3L * qInvL + q3R * qInvR);
    const double Yeta_A = 0.5 * (YetaL + YetaR);
    const double Xeta_A = 0.5 * (XetaL + XetaR);
    const double p = h_A - c->half_g * h2_A;
    *F1 = Yeta_A * hu_A - Xeta_A * hv_A;
    *F2 = Yeta_A * (hu_A * u_A + p) - Xeta_A * hv_A * u_A;
    *F3 = Yeta_A * (hu_A * v_A) - Xeta_A * (hv_A * v_A + p);
}
static inline void Gvol(const oconst* c, double q1L, double q2L, double q3L, double qInvL, double q1R, double q2R,
                        double q3R, double qInvR, double YxiL, double YxiR, double XxiL, double XxiR, double* G1,
                        double* G2, double* G3) {
    const double h_A = c->fourth_g * (q1L + q1R) * (q1L + q1R);
    const double h2_A = 0.5 * (q1L * q1L + q1R * q1R);
    const double hu_A = 0.5 * (q2L + q2R);
    const double hv_A = 0.5 * (q3L + q3R);
    const double u_A = 0.5 * (q2L * qInvL + q2R * qInvR);
    const double v_A = 0.5 * (q3L * qInvL + q3R * qInvR);
    const double Yxi_A = 0.5 * (YxiL + YxiR);
    const double Xxi_A = 0.5 * (XxiL + XxiR);
    const double p = h_A - c->half_g * h2_A;
    *G1 = -Yxi_A * hu_A + Xxi_A * hv_A;
    *G2 = -Yxi_A * (hu_A * u_A + p) + Xxi_A * hv_A * u_A;
    *G3 = -Yxi_A * (hu_A * v_A) + Xxi_A * (hv_A * v_A + p);
}

/* --- okl/DG/VolumeKernelFluxDiffV99.okl:60-218 ----------------------------- */
static void volume_fluxdiff(const oconst* c, int K, const double* Jac, const double* Yxi, const double* Yeta,
                            const double* Xxi, const double* Xeta, const double* Q, const double* D,
                            const double* Bx, const double* By, double* Qt) {
    const int ngl = c->ngl, n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e) {
        double sQ1[64], sQ2[64], sQ3[64], sI[64], sYe[64], sYx[64], sXe[64], sXx[64];
        for (int id = 0; id < n2; ++id) {
            const long xid = (long)e * n2 + id, Fid = (long)e * n2 * NEQ + id;
            sYe[id] = Yeta[xid]; sYx[id] = Yxi[xid]; sXe[id] = Xeta[xid]; sXx[id] = Xxi[xid];
            sQ1[id] = Q[Fid]; sQ2[id] = Q[Fid + n2]; sQ3[id] = Q[Fid + 2 * n2];
            sI[id] = (Q[Fid] > 0) ? 1.0 / Q[Fid] : 0.0;
        }
        for (int i = 0; i < ngl; ++i)      /* eta index (slow) */
            for (int j = 0; j < ngl; ++j) { /* xi index (fast)  */
                const int ij = i * ngl + j;
                const long id = (long)e * n2 * NEQ + ij, xid = (long)e * n2 + ij;
                double d1 = 0, d2 = 0, d3 = 0;
                for (int l = 0; l < ngl; ++l) {
                    const double djl = D[j * ngl + l];
                    const int il = i * ngl + l;
                    double f1, f2, f3;
                    Fvol(c, sQ1[ij], sQ2[ij], sQ3[ij], sI[ij], sQ1[il], sQ2[il], sQ3[il], sI[il], sYe[ij], sYe[il],
                         sXe[ij], sXe[il], &f1, &f2, &f3);
                    d1 += djl * f1; d2 += djl * f2; d3 += djl * f3;
                }
                for (int l = 0; l < ngl; ++l) {
                    const double dil = D[i * ngl + l];
                    const int lj = l * ngl + j;
                    double g1, g2, g3;
                    Gvol(c, sQ1[ij], sQ2[ij], sQ3[ij], sI[ij], sQ1[lj], sQ2[lj], sQ3[lj], sI[lj], sYx[ij], sYx[lj],
                         sXx[ij], sXx[lj], &g1, &g2, &g3);
                    d1 += dil * g1; d2 += dil * g2; d3 += dil * g3;
                }
                const double J = Jac[xid];
                Qt[id] = -J * d1;
                Qt[id + n2] = -J * d2 - c->g_const * sQ1[ij] * Bx[xid];
                Qt[id + 2 * n2] = -J * d3 - c->g_const * sQ1[ij] * By[xid];
            }
    }
}

/* --- Riemann solvers ------------------------------------------------------- */
/* variant 0: okl/RiemannSolvers/calcESFlux.okl:17-215
 * variant 3: okl/RiemannSolvers/calcESFluxRotated.okl:17-214
 * variant 2: okl/RiemannSolvers/calcLFTypeESFlux.okl:17-195, repaired: the
 *            reference call site passes EdgeReversed which that kernel does
 *            not declare (src/deviceclass.cpp:1004), and it reads qR without
 *            reversing the right element's node order; here both are fixed
 *            exactly as in variants 0/3.                                    */
static void es_flux_point(const oconst* c, int variant, double nx, double ny, double hL, double huL, double hvL,
                          double hR, double huR, double hvR, double bL, double bR, double* NF) {
    const double tol = c->PosPresTOL, g = c->g_const;
    double uL, vL, uR, vR;
    if (variant == 0) {
        if (hL >= tol) { uL = huL / hL; vL = hvL / hL; } else { hL = 0.0; uL = 0.0; vL = 0.0; }
        if (hR >= tol) { uR = huR / hR; vR = hvR / hR; } else { hR = 0.0; uR = 0.0; vR = 0.0; }
        const double avgH = 0.5 * (hL + hR), avgH2 = 0.5 * (hL * hL + hR * hR);
        const double avgU = 0.5 * (uL + uR), avgV = 0.5 * (vL + vR);
        const double normV = avgU * nx + avgV * ny;
        NF[0] = avgH * normV;
        NF[1] = avgH * avgU * normV + (0.5 * g * avgH2) * nx;
        NF[2] = avgH * avgV * normV + (0.5 * g * avgH2) * ny;
        if (c->ES) {
            const double cL = g * hL, cR = g * hR;
            const double avgC = sqrt(fabs(0.5 * (cL + cR)));
            const double q1L = g * (hL + bL) - 0.5 * uL * uL - 0.5 * vL * vL;
            const double q1R = g * (hR + bR) - 0.5 * uR * uR - 0.5 * vR * vR;
            const double j1 = q1R - q1L, j2 = uR - uL, j3 = vR - vL;
            const double R11 = 1.0, R12 = 0.0, R13 = 1.0;
            const double R21 = avgU + nx * avgC, R22 = ny, R23 = avgU - nx * avgC;
            const double R31 = avgV + ny * avgC, R32 = nx, R33 = avgV - ny * avgC;
            const double SL11 = 0.5 / g * fabs(nx * avgU + ny * avgV + avgC);
            const double SL22 = fabs(avgH * (nx * avgU + ny * avgV));
            const double SL33 = 0.5 / g * fabs(nx * avgU + ny * avgV - avgC);
            const double RSL11 = R11 * SL11, RSL12 = 0.0, RSL13 = R13 * SL33;
            const double RSL21 = R21 * SL11, RSL22 = R22 * SL22, RSL23 = R23 * SL33;
            const double RSL31 = R31 * SL11, RSL32 = R32 * SL22, RSL33 = R33 * SL33;
            const double M11 = RSL11 * R11 + RSL12 * R12 + RSL13 * R13;
            const double M12 = RSL11 * R21 + RSL12 * R22 + RSL13 * R23;
            const double M13 = RSL11 * R31 + RSL12 * R32 + RSL13 * R33;
            const double M21 = RSL21 * R11 + RSL22 * R12 + RSL23 * R13;
            const double M22 = RSL21 * R21 + RSL22 * R22 + RSL23 * R23;
            const double M23 = RSL21 * R31 + RSL22 * R32 + RSL23 * R33;
            const double M31 = RSL31 * R11 + RSL32 * R12 + RSL33 * R13;
            const double M32 = RSL31 * R21 + RSL32 * R22 + RSL33 * R23;
            const double M33 = RSL31 * R31 + RSL32 * R32 + RSL33 * R33;
            NF[0] += -0.5 * (M11 * j1 + M12 * j2 + M13 * j3);
            NF[1] += -0.5 * (M21 * j1 + M22 * j2 + M23 * j3);
            NF[2] += -0.5 * (M31 * j1 + M32 * j2 + M33 * j3);
        }
    } else if (variant == 3) {
        if (hL > tol) { uL = huL / hL; vL = hvL / hL; } else { uL = 0.0; vL = 0.0; }
        if (hR > tol) { uR = huR / hR; vR = hvR / hR; } else { uR = 0.0; vR = 0.0; }
        const double vLn = nx * uL + ny * vL, vLt = -ny * uL + nx * vL;
        const double vRn = nx * uR + ny * vR, vRt = -ny * uR + nx * vR;
        const double avgH = 0.5 * (hL + hR), avgH2 = 0.5 * (hL * hL + hR * hR);
        const double avgU = 0.5 * (vLn + vRn), avgV = 0.5 * (vLt + vRt);
        double N0 = avgH * avgU;
        double N1 = avgH * avgU * avgU + (0.5 * g * avgH2);
        double N2 = avgH * avgV * avgU;
        if (c->ES) {
            const double cL = g * hL, cR = g * hR;
            const double avgC = sqrt(fabs(0.5 * (cL + cR)));
            const double q1L = g * (hL + bL) - 0.5 * vLn * vLn - 0.5 * vLt * vLt;
            const double q1R = g * (hR + bR) - 0.5 * vRn * vRn - 0.5 * vRt * vRt;
            const double j1 = q1R - q1L, j2 = vRn - vLn, j3 = vRt - vLt;
            const double R11 = 1.0, R12 = 0.0, R13 = 1.0;
            const double R21 = avgU + avgC, R22 = 0.0, R23 = avgU - avgC;
            const double R31 = avgV, R32 = 1.0, R33 = avgV;
            const double SL11 = 0.5 / g * fabs(avgU + avgC);
            const double SL22 = fabs(avgH * avgU);
            const double SL33 = 0.5 / g * fabs(avgU - avgC);
            const double RSL11 = R11 * SL11, RSL12 = 0.0, RSL13 = R13 * SL33;
            const double RSL21 = R21 * SL11, RSL22 = R22 * SL22, RSL23 = R23 * SL33;
            const double RSL31 = R31 * SL11, RSL32 = R32 * SL22, RSL33 = R33 * SL33;
            const double M11 = RSL11 * R11 + RSL12 * R12 + RSL13 * R13;
            const double M12 = RSL11 * R21 + RSL12 * R22 + RSL13 * R23;
            const double M13 = RSL11 * R31 + RSL12 * R32 + RSL13 * R33;
            const double M21 = RSL21 * R11 + RSL22 * R12 + RSL23 * R13;
            const double M22 = RSL21 * R21 + RSL22 * R22 + RSL23 * R23;
            const double M23 = RSL21 * R31 + RSL22 * R32 + RSL23 * R33;
            const double M31 = RSL31 * R11 + RSL32 * R12 + RSL33 * R13;
            const double M32 = RSL31 * R21 + RSL32 * R22 + RSL33 * R23;
            const double M33 = RSL31 * R31 + RSL32 * R32 + RSL33 * R33;
            N0 += -0.5 * (M11 * j1 + M12 * j2 + M13 * j3);
            N1 += -0.5 * (M21 * j1 + M22 * j2 + M23 * j3);
            N2 += -0.5 * (M31 * j1 + M32 * j2 + M33 * j3);
        }
        NF[0] = N0;
        NF[1] = nx * N1 - ny * N2;
        NF[2] = ny * N1 + nx * N2;
    } else { /* variant 2 */
        if (hL > tol) { uL = huL / hL; vL = hvL / hL; } else { uL = 0.0; vL = 0.0; }
        if (hR > tol) { uR = huR / hR; vR = hvR / hR; } else { uR = 0.0; vR = 0.0; }
        const double avgH = 0.5 * (hL + hR), avgH2 = 0.5 * (hL * hL + hR * hR);
        const double avgU = 0.5 * (uL + uR), avgV = 0.5 * (vL + vR);
        const double normV = avgU * nx + avgV * ny;
        NF[0] = avgH * normV;
        NF[1] = avgH * avgU * normV + (0.5 * g * avgH2) * nx;
        NF[2] = avgH * avgV * normV + (0.5 * g * avgH2) * ny;
        if (c->ES) {
            const double cL = (hL > tol) ? sqrt(g * hL) : 0.0;
            const double cR = (hR > tol) ? sqrt(g * hR) : 0.0;
            const double q1L = g * (hL + bL) - 0.5 * uL * uL - 0.5 * vL * vL;
            const double q1R = g * (hR + bR) - 0.5 * uR * uR - 0.5 * vR * vR;
            const double j1 = q1R - q1L, j2 = uR - uL, j3 = vR - vL;
            const double H11 = 1.0, H12 = avgU, H13 = avgV;
            const double H21 = avgU, H22 = g * avgH + avgU * avgU, H23 = avgU * avgV;
            const double H31 = avgV, H32 = avgU * avgV, H33 = g * avgH + avgV * avgV;
            const double lL = cL + dmax(fabs(uL), fabs(vL));
            const double lR = cR + dmax(fabs(uR), fabs(vR));
            const double lam = dmax(lL, lR) / g;
            NF[0] += -0.5 * lam * (H11 * j1 + H12 * j2 + H13 * j3);
            NF[1] += -0.5 * lam * (H21 * j1 + H22 * j2 + H23 * j3);
            NF[2] += -0.5 * lam * (H31 * j1 + H32 * j2 + H33 * j3);
        }
    }
}

static void num_fluxes(const oconst* c, int variant, int F, const int* EdgeReversed, const double* nxa,
                       const double* nya, const double* Scal, const double* qL, const double* qR, const double* BL,
                       const double* BR, double* SP) {
    const int ngl = c->ngl;
#pragma omp parallel for schedule(static)
    for (int ifa = 0; ifa < F; ++ifa)
        for (int i = 0; i < ngl; ++i) {
            const long ex = (long)ifa * ngl + i, eid = (long)ifa * ngl * NEQ + i;
            const int rev = EdgeReversed[ifa];
            const int ir = (1 - rev) * (ngl - 1 - i) + rev * i;
            const long eidR = (long)ifa * ngl * NEQ + ir, exR = (long)ifa * ngl + ir;
            double NF[3];
            es_flux_point(c, variant, nxa[ex], nya[ex], qL[eid], qL[eid + ngl], qL[eid + 2 * ngl], qR[eidR],
                          qR[eidR + ngl], qR[eidR + 2 * ngl], BL[ex], BR[exR], NF);
            const double s = Scal[ex];
            SP[eid] = s * c->geomFace * NF[0];
            SP[eid + ngl] = s * c->geomFace * NF[1];
            SP[eid + 2 * ngl] = s * c->geomFace * NF[2];
        }
}

/* --- okl/DG/SurfaceKernel.okl:17-142 (DBSurf1/2 are zero: DiscBottom=0) --- */
static void surface_lift(int ngl, int K, const double* Jac, const int* MS, const int* OR, const int* E2E,
                         const double* FS, double* Qt) {
    const int n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int ie = 0; ie < K; ++ie) {
        for (int pass = 0; pass < 2; ++pass)
            for (int is = 0; is < 2; ++is)
                for (int j = 0; j < ngl; ++j) {
                    const int iside = 2 * is + pass;
                    const int ifa = E2E[ie * 4 + iside] - 1;
                    const int ro = OR[ie * 4 + iside];
                    const int inc = ro * j + (1 - ro) * (ngl - 1 - j);
                    const long fl = (long)ifa * ngl * NEQ + inc;
                    long xid, id;
                    if (pass == 0) {
                        xid = (long)ie * n2 + is * (n2 - ngl) + j;
                        id = (long)ie * n2 * NEQ + is * (n2 - ngl) + j;
                    } else {
                        xid = (long)ie * n2 + (long)j * ngl + (1 - is) * (ngl - 1);
                        id = (long)ie * n2 * NEQ + (1 - is) * (ngl - 1) + (long)j * ngl;
                    }
                    const int ms = MS[ie * 4 + iside];
                    const double J = Jac[xid];
                    const double db = 0.0;
                    Qt[id] += -ms * FS[fl] * J;
                    Qt[id + n2] += -ms * J * FS[fl + ngl] + J * db;
                    Qt[id + 2 * n2] += -ms * J * FS[fl + 2 * ngl] + J * db;
                }
    }
}

/* --- okl/DG/FindLambdaMax.okl:17-100 + host max (src/deviceclass.cpp:899-908) */
static double lambda_max(const oconst* c, int K, const double* Q) {
    const int ngl = c->ngl, n2 = ngl * ngl;
    double gl = 0.0;
#pragma omp parallel for reduction(max : gl) schedule(static)
    for (int e = 0; e < K; ++e) {
        double lm = 0.0;
        for (int id = 0; id < n2; ++id) {
            const long Fid = (long)e * n2 * NEQ + id;
            const double h = Q[Fid];
            const double inv = (h > c->PosPresTOL) ? 1.0 / h : 0.0;
            const double cc = sqrt(c->g_const * h);
            const double u = Q[Fid + n2] * inv, v = Q[Fid + 2 * n2] * inv;
            lm = dmax(lm, cc + dmax(fabs(u), fabs(v)));
        }
        gl = fmax(gl, lm);
    }
    return gl;
}

/* --- okl/ShockCapturing/ShockCapturing.okl:17-234 ------------------------ */
static void shock_capturing(const oconst* c, int K, const double* Q, const double* b, const double* Vinv,
                            double* ViscPara) {
    const int ngl = c->ngl, n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e) {
        double sM[64], sV[64], s1[64];
        for (int i = 0; i < ngl; ++i)
            for (int j = 0; j < ngl; ++j) {
                const long Fid = (long)e * n2 * NEQ + j * ngl + i, Xid = (long)e * n2 + j * ngl + i;
                sV[i * ngl + j] = Vinv[j * ngl + i];
                sM[i * ngl + j] = b[Xid] + Q[Fid];
            }
        for (int i = 0; i < ngl; ++i)
            for (int j = 0; j < ngl; ++j) {
                double a = 0.0;
                for (int l = 0; l < ngl; ++l) a += sV[l * ngl + i] * sM[l * ngl + j];
                s1[i * ngl + j] = a;
            }
        for (int i = 0; i < ngl; ++i)
            for (int j = 0; j < ngl; ++j) {
                double a = 0.0;
                for (int l = 0; l < ngl; ++l) a += s1[i * ngl + l] * sV[l * ngl + j];
                sM[i * ngl + j] = a;
            }
        const int N = ngl - 1;
        double z1 = 0, n1 = 0, z2 = 0, n2s = 0;
        for (int i = 0; i < N; ++i)
            z1 += sM[i * ngl + N] * sM[i * ngl + N] + sM[N * ngl + i] * sM[N * ngl + i];
        z1 += sM[N * ngl + N] * sM[N * ngl + N];
        for (int i = 0; i < N - 1; ++i)
            z2 += sM[i * ngl + N - 1] * sM[i * ngl + N - 1] + sM[(N - 1) * ngl + i] * sM[(N - 1) * ngl + i];
        z2 += sM[(N - 1) * ngl + N - 1] * sM[(N - 1) * ngl + N - 1];
        for (int i = 0; i < ngl; ++i)
            for (int j = 0; j < ngl; ++j) n1 += sM[i * ngl + j] * sM[i * ngl + j];
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) n2s += sM[i * ngl + j] * sM[i * ngl + j];
        const double t1 = (n1 < c->ZeroTOL) ? 0.0 : z1 / n1;
        const double t2 = (n1 < c->ZeroTOL) ? 0.0 : z2 / n2s;
        double sig = (t1 < t2) ? t2 : t1;
        sig = log10(sig);
        double vs;
        if (c->sigmaMin >= sig) vs = 0.0;
        else if (c->sigmaMax >= sig) {
            const double delta =
                1.0 + sin(c->PI * (sig - 0.5 * (c->sigmaMax + c->sigmaMin)) / (c->sigmaMax - c->sigmaMin));
            vs = c->eps0 * 0.5 * delta;
        } else vs = c->eps0;
        ViscPara[e] = vs;
    }
}

/* --- okl/BR1_Gradient/calcNumFluxesGradient.okl:16-135 -------------------- */
static void num_fluxes_gradient(const oconst* c, int F, const int* EdgeData, const double* nxa, const double* nya,
                                const double* Scal, const double* qL, const double* qR, double* SGX, double* SGY) {
    const int ngl = c->ngl;
#pragma omp parallel for schedule(static)
    for (int ifa = 0; ifa < F; ++ifa)
        for (int i = 0; i < ngl; ++i) {
            const int cpuL = EdgeData[8 * ifa + 5], cpuR = EdgeData[8 * ifa + 6];
            const long eid = (long)ifa * ngl * NEQ + i, gid = (long)ifa * ngl * 2 + i, ex = (long)ifa * ngl + i;
            const double nx = nxa[ex], ny = nya[ex], sc = Scal[ex];
            double hL, huL, hvL, hR, huR, hvR;
            if (cpuL == -1) { hL = qR[eid]; huL = qR[eid + ngl]; hvL = qR[eid + 2 * ngl]; }
            else { hL = qL[eid]; huL = qL[eid + ngl]; hvL = qL[eid + 2 * ngl]; }
            if (cpuR == -1) { hR = qL[eid]; huR = qL[eid + ngl]; hvR = qL[eid + 2 * ngl]; }
            else { hR = qR[eid]; huR = qR[eid + ngl]; hvR = qR[eid + 2 * ngl]; }
            const double iL = (hL > c->PosPresTOL) ? 1.0 / hL : 0.0;
            const double iR = (hR > c->PosPresTOL) ? 1.0 / hR : 0.0;
            const double uL = huL * iL, uR = huR * iR, vL = hvL * iL, vR = hvR * iR;
            SGX[gid] = nx * sc * c->geomFace * 0.5 * (uL + uR);
            SGX[gid + ngl] = nx * sc * c->geomFace * 0.5 * (vL + vR);
            SGY[gid] = ny * sc * c->geomFace * 0.5 * (uL + uR);
            SGY[gid + ngl] = ny * sc * c->geomFace * 0.5 * (vL + vR);
        }
}

/* --- okl/BR1_Gradient/calcGradient.okl:18-156 ----------------------------- */
static void calc_gradient(const oconst* c, int K, const double* Jac, const double* Yxi, const double* Yeta,
                          const double* Xxi, const double* Xeta, const double* Q, const double* Dh, double* GX,
                          double* GY) {
    const int ngl = c->ngl, n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e) {
        double su[64], sv[64], sD[64];
        for (int i = 0; i < ngl; ++i)
            for (int j = 0; j < ngl; ++j) {
                const long Fid = (long)e * n2 * NEQ + j * ngl + i;
                sD[i * ngl + j] = Dh[j * ngl + i];
                const double h = Q[Fid];
                const double inv = (h > c->PosPresTOL) ? 1.0 / h : 0.0;
                su[i * ngl + j] = Q[Fid + n2] * inv;
                sv[i * ngl + j] = Q[Fid + 2 * n2] * inv;
            }
        for (int i = 0; i < ngl; ++i)
            for (int j = 0; j < ngl; ++j) {
                const long xid = (long)e * n2 + j * ngl + i;
                double uxi = 0, ueta = 0, vxi = 0, veta = 0;
                for (int l = 0; l < ngl; ++l) {
                    uxi += sD[l * ngl + i] * su[l * ngl + j];
                    ueta += sD[l * ngl + j] * su[i * ngl + l];
                    vxi += sD[l * ngl + i] * sv[l * ngl + j];
                    veta += sD[l * ngl + j] * sv[i * ngl + l];
                }
                const long id = (long)e * n2 * 2 + j * ngl + i;
                const double J = Jac[xid];
                const double ux = Yeta[xid] * uxi - Yxi[xid] * ueta;
                const double vx = Yeta[xid] * vxi - Yxi[xid] * veta;
                const double uy = -Xeta[xid] * uxi + Xxi[xid] * ueta;
                const double vy = -Xeta[xid] * vxi + Xxi[xid] * veta;
                GX[id] = J * ux; GX[id + n2] = J * vx;
                GY[id] = J * uy; GY[id + n2] = J * vy;
            }
    }
}

/* Lift of a 2-component face quantity into [K][2][n][n] (+= s*J*F):
 * okl/BR1_Gradient/SurfaceKernelGradient.okl:16-150 (sign +) and
 * okl/ViscoseParts/SurfaceKernelVisc.okl:17-144 (sign -, into Qt eqs 1,2). */
static void surface_lift_grad(int ngl, int K, const double* Jac, const int* MS, const int* OR, const int* E2E,
                              const double* UX, const double* UY, double* GX, double* GY) {
    const int n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int ie = 0; ie < K; ++ie)
        for (int pass = 0; pass < 2; ++pass)
            for (int is = 0; is < 2; ++is)
                for (int j = 0; j < ngl; ++j) {
                    const int iside = 2 * is + pass;
                    const int ifa = E2E[ie * 4 + iside] - 1;
                    const int ro = OR[ie * 4 + iside];
                    const int inc = ro * j + (1 - ro) * (ngl - 1 - j);
                    const long fl = (long)ifa * ngl * 2 + inc;
                    long xid, id;
                    if (pass == 0) {
                        xid = (long)ie * n2 + is * (n2 - ngl) + j;
                        id = (long)ie * n2 * 2 + is * (n2 - ngl) + j;
                    } else {
                        xid = (long)ie * n2 + (long)j * ngl + (1 - is) * (ngl - 1);
                        id = (long)ie * n2 * 2 + (1 - is) * (ngl - 1) + (long)j * ngl;
                    }
                    const int ms = MS[ie * 4 + iside];
                    const double J = Jac[xid];
                    if (pass == 0) GX[id] += ms * UX[fl] * J;
                    else GX[id] += ms * J * UX[fl];
                    GX[id + n2] += ms * J * UX[fl + ngl];
                    GY[id] += ms * J * UY[fl];
                    GY[id + n2] += ms * J * UY[fl + ngl];
                }
}

static void surface_lift_visc(int ngl, int K, const double* Jac, const int* MS, const int* OR, const int* E2E,
                              const double* FS, double* Qt) {
    const int n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int ie = 0; ie < K; ++ie)
        for (int pass = 0; pass < 2; ++pass)
            for (int is = 0; is < 2; ++is)
                for (int j = 0; j < ngl; ++j) {
                    const int iside = 2 * is + pass;
                    const int ifa = E2E[ie * 4 + iside] - 1;
                    const int ro = OR[ie * 4 + iside];
                    const int inc = ro * j + (1 - ro) * (ngl - 1 - j);
                    const long fl = (long)ifa * ngl * 2 + inc;
                    long xid, id;
                    if (pass == 0) {
                        xid = (long)ie * n2 + is * (n2 - ngl) + j;
                        id = (long)ie * n2 * NEQ + is * (n2 - ngl) + j;
                    } else {
                        xid = (long)ie * n2 + (long)j * ngl + (1 - is) * (ngl - 1);
                        id = (long)ie * n2 * NEQ + (1 - is) * (ngl - 1) + (long)j * ngl;
                    }
                    const int ms = MS[ie * 4 + iside];
                    const double J = Jac[xid];
                    Qt[id + n2] += -ms * J * FS[fl];
                    Qt[id + 2 * n2] += -ms * J * FS[fl + ngl];
                }
}

/* --- okl/BR1_Gradient/scaleGradient.okl:17-60 ----------------------------- */
static void scale_gradient(int ngl, int K, const double* Q, double* GX, double* GY) {
    const int n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e)
        for (int id = 0; id < n2; ++id) {
            const double h = Q[(long)e * n2 * NEQ + id];
            const long g = (long)e * n2 * 2 + id;
            GX[g] = h * GX[g]; GX[g + n2] = h * GX[g + n2];
            GY[g] = h * GY[g]; GY[g + n2] = h * GY[g + n2];
        }
}

/* --- okl/BR1_Gradient/CollectEdgeDataGradient.okl:17-194 ------------------
 * Boundary faces leave the R/Y slots as they were (never read downstream,
 * the viscous flux is zero there); here they are zeroed.                    */
static void collect_edge_gradient(int ngl, int F, const int* EdgeData, const double* GX, const double* GY,
                                  const double* VP, double* VPL, double* VPR, double* GXL, double* GXR, double* GYL,
                                  double* GYR) {
    const int n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int ifa = 0; ifa < F; ++ifa)
        for (int i = 0; i < ngl; ++i) {
            const int iel = EdgeData[8 * ifa], ier = EdgeData[8 * ifa + 1];
            const int isl = EdgeData[8 * ifa + 2], isr = EdgeData[8 * ifa + 3];
            const int rev = EdgeData[8 * ifa + 4];
            const int cpuL = EdgeData[8 * ifa + 5], cpuR = EdgeData[8 * ifa + 6];
            const int inc = (rev == 0) ? (ngl - 1) - i : i;
            const long eid = (long)ifa * ngl * 2 + i;
            double XL[2] = {0, 0}, XR[2] = {0, 0}, YL[2] = {0, 0}, YR[2] = {0, 0};
            if (i == 0) { VPL[ifa] = 0.0; VPR[ifa] = 0.0; }
            if (cpuL == 0) {
                const long id = trace_index(iel, isl, i, ngl, 2);
                XL[0] = GX[id]; XL[1] = GX[id + n2]; YL[0] = GY[id]; YL[1] = GY[id + n2];
                if (i == 0) VPL[ifa] = VP[iel];
            }
            if (cpuR == 0) {
                const long id = trace_index(ier, isr, inc, ngl, 2);
                XR[0] = GX[id]; XR[1] = GX[id + n2]; YR[0] = GY[id]; YR[1] = GY[id + n2];
                if (i == 0) VPR[ifa] = VP[ier];
            }
            if (cpuL == -1) {
                if (i == 0) { VPL[ifa] = VP[ier]; VPR[ifa] = VP[ier]; }
                XL[0] = 0.0; XL[1] = 0.0;
            }
            if (cpuR == -1) {
                if (i == 0) { VPL[ifa] = VP[iel]; VPR[ifa] = VP[iel]; }
                XL[0] = 0.0; XL[1] = 0.0;
            }
            GXL[eid] = XL[0]; GXL[eid + ngl] = XL[1];
            GXR[eid] = XR[0]; GXR[eid + ngl] = XR[1];
            GYL[eid] = YL[0]; GYL[eid + ngl] = YL[1];
            GYR[eid] = YR[0]; GYR[eid + ngl] = YR[1];
        }
}

/* --- okl/ViscoseParts/VolumeKernelViscose.okl:17-150 ---------------------- */
static void volume_viscous(const oconst* c, int K, const double* Jac, const double* Yxi, const double* Yeta,
                           const double* Xxi, const double* Xeta, const double* GX, const double* GY,
                           const double* Ds, const double* VP, double* Qt) {
    const int ngl = c->ngl, n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e) {
        double sF2[64], sF3[64], sG2[64], sG3[64], sD[64];
        const double eps = VP[e];
        for (int i = 0; i < ngl; ++i)
            for (int j = 0; j < ngl; ++j) {
                const long xid = (long)e * n2 + j * ngl + i, Fid = (long)e * n2 * 2 + j * ngl + i;
                sD[i * ngl + j] = Ds[j * ngl + i];
                const double F2 = eps * GX[Fid], F3 = eps * GX[Fid + n2];
                const double G2 = eps * GY[Fid], G3 = eps * GY[Fid + n2];
                sF2[i * ngl + j] = Yeta[xid] * F2 - Xeta[xid] * G2;
                sG2[i * ngl + j] = -Yxi[xid] * F2 + Xxi[xid] * G2;
                sF3[i * ngl + j] = Yeta[xid] * F3 - Xeta[xid] * G3;
                sG3[i * ngl + j] = -Yxi[xid] * F3 + Xxi[xid] * G3;
            }
        for (int j = 0; j < ngl; ++j)
            for (int i = 0; i < ngl; ++i) {
                double d2 = 0, d3 = 0;
                for (int l = 0; l < ngl; ++l) {
                    d2 += sD[l * ngl + i] * sF2[l * ngl + j];
                    d2 += sD[l * ngl + j] * sG2[i * ngl + l];
                    d3 += sD[l * ngl + i] * sF3[l * ngl + j];
                    d3 += sD[l * ngl + j] * sG3[i * ngl + l];
                }
                const long id = (long)e * n2 * NEQ + j * ngl + i, xid = (long)e * n2 + j * ngl + i;
                const double J = Jac[xid];
                Qt[id + n2] += J * d2;
                Qt[id + 2 * n2] += J * d3;
            }
    }
}

/* --- okl/ViscoseParts/calcNumFluxesViscose.okl:17-107 --------------------- */
static void num_fluxes_viscous(const oconst* c, int F, const int* EdgeData, const double* nxa, const double* nya,
                               const double* Scal, const double* VPL, const double* VPR, const double* XL,
                               const double* XR, const double* YL, const double* YR, double* SP) {
    const int ngl = c->ngl;
#pragma omp parallel for schedule(static)
    for (int ifa = 0; ifa < F; ++ifa)
        for (int i = 0; i < ngl; ++i) {
            const long ex = (long)ifa * ngl + i, eid = (long)ifa * ngl * 2 + i;
            const int cpuL = EdgeData[8 * ifa + 5], cpuR = EdgeData[8 * ifa + 6];
            const double nx = nxa[ex], ny = nya[ex], sc = Scal[ex];
            const double f2L = nx * XL[eid] + ny * YL[eid], f2R = nx * XR[eid] + ny * YR[eid];
            const double f3L = nx * XL[eid + ngl] + ny * YL[eid + ngl];
            const double f3R = nx * XR[eid + ngl] + ny * YR[eid + ngl];
            double N0, N1;
            if (cpuL == -1 || cpuR == -1) { N0 = 0.0; N1 = 0.0; }
            else {
                N0 = 0.5 * dmax(VPL[ifa], VPR[ifa]) * (f2L + f2R);
                N1 = 0.5 * dmax(VPL[ifa], VPR[ifa]) * (f3L + f3R);
            }
            SP[eid] = -sc * c->geomFace * N0;
            SP[eid + ngl] = -sc * c->geomFace * N1;
        }
}

/* --- okl/Positivity/PosPres.okl:17-223 ----------------------------------- */
static void pos_pres(const oconst* c, int K, const double* EleSizes, const double* GLw, const double* Jac,
                     double* Q) {
    const int ngl = c->ngl, n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e) {
        double hmin = 0.0, ha = 0.0, hua = 0.0, hva = 0.0;
        for (int l = 0; l < ngl; ++l)
            for (int k = 0; k < ngl; ++k) {
                const long xid = (long)e * n2 + k * ngl + l, Fid = (long)e * n2 * NEQ + k * ngl + l;
                const double w = GLw[l] * GLw[k] / Jac[xid];
                ha += Q[Fid] * w;
                hua += Q[Fid + n2] * w;
                hva += Q[Fid + 2 * n2] * w;
                hmin = dmin(hmin, Q[Fid]);
            }
        ha = ha / EleSizes[e];
        if (fabs(ha) < c->ZeroTOL) ha = 0.0;
        const double theta = (ha == hmin) ? 1.0 : dmin(1.0, ha / (ha - hmin));
        hua = hua / EleSizes[e];
        hva = hva / EleSizes[e];
        for (int id = 0; id < n2; ++id) {
            const long Fid = (long)e * n2 * NEQ + id;
            const double h = Q[Fid], hu = Q[Fid + n2], hv = Q[Fid + 2 * n2];
            if (hmin < 0.0) {
                double hn = 0.0, hun = 0.0, hvn = 0.0;
                if (ha > 0.0) {
                    hn = fabs(theta * (h - ha) + ha);
                    if (hn > c->PosPresTOL) {
                        hun = theta * (hu - hua) + hua;
                        hvn = theta * (hv - hva) + hva;
                    }
                }
                if (ha < 0.0) { hn = -1.0 / 0.0; hun = 0.0; hvn = 0.0; }
                Q[Fid] = hn; Q[Fid + n2] = hun; Q[Fid + 2 * n2] = hvn;
            } else if (h < c->PosPresTOL) {
                Q[Fid + n2] = 0.0;
                Q[Fid + 2 * n2] = 0.0;
            }
        }
    }
}

/* --- okl/PartialDryTreatment/FindDryElements.okl:16-63 -------------------- */
static void find_dry(const oconst* c, int K, const double* Q, int* dry) {
    const int ngl = c->ngl, n2 = ngl * ngl;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e) {
        double mh = 1.0;
        for (int k = 0; k < ngl; ++k)
            for (int l = 0; l < ngl; ++l) mh = fmin(Q[(long)e * n2 * NEQ + k * ngl + l], mh);
        dry[e] = mh < c->PosPresTOL ? 1 : 0;
    }
}

/* --- okl/PartialDryTreatment/VolumeKernelFD.okl:33-343: momentum volume
 * terms of partly dry elements, overwriting Qt[hu], Qt[hv] there (called
 * right after the volume kernel, src/deviceclass.cpp:987-991).  Row i is
 * eta, column j is xi; a difference uses a neighbour only where it is wet. */
static void volume_partial_dry(const oconst* c, int K, const double* Jac, const double* Yxi, const double* Yeta,
                               const double* Xxi, const double* Xeta, const double* Q, const int* dry,
                               const double* Dc, const double* Dup, const double* Ddn, const double* B, double* Qt) {
    const int n = c->ngl, n2 = n * n;
    const double tol = c->PosPresTOL, g = c->g_const;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e) {
        if (dry[e] != 1) continue;
        const double* H = Q + (long)e * n2 * NEQ; /* h of the element, [i][j] */
        const double* b = B + (long)e * n2;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const int id = i * n + j;
                const double h = H[id], bb = b[id];
                const double xm = j > 0 ? H[id - 1] : 0.0, xp = j < n - 1 ? H[id + 1] : 0.0;
                const double ym = i > 0 ? H[id - n] : 0.0, yp = i < n - 1 ? H[id + n] : 0.0;
                /* F2_2 = G3_2 = g h; the derivatives of F and G coincide */
                double dFxi = 0.0, dFeta = 0.0, dBxi = 0.0, dBeta = 0.0;
                if (h > tol) {
                    if (j == 0 && xp > tol) {
                        dFxi = Dup[j * n + 0] * (g * h) + Dup[j * n + 1] * (g * H[id + 1]);
                        dBxi = Dup[j * n + 0] * bb + Dup[j * n + 1] * b[id + 1];
                    }
                    if (j == n - 1 && xm > tol) {
                        dFxi = Ddn[j * n + n - 2] * (g * H[id - 1]) + Ddn[j * n + n - 1] * (g * h);
                        dBxi = Ddn[j * n + n - 2] * b[id - 1] + Ddn[j * n + n - 1] * bb;
                    }
                    if (j > 0 && j < n - 1) {
                        if (xp > tol && xm > tol) {
                            dFxi = Dc[j * n + j - 1] * (g * H[id - 1]) + Dc[j * n + j + 1] * (g * H[id + 1]);
                            dBxi = Dc[j * n + j - 1] * b[id - 1] + Dc[j * n + j + 1] * b[id + 1];
                        } else if (xp > tol) {
                            dFxi = Dup[j * n + j] * (g * h) + Dup[j * n + j + 1] * (g * H[id + 1]);
                            dBxi = Dup[j * n + j] * bb + Dup[j * n + j + 1] * b[id + 1];
                        } else if (xm > tol) {
                            dFxi = Ddn[j * n + j - 1] * (g * H[id - 1]) + Ddn[j * n + j] * (g * h);
                            dBxi = Ddn[j * n + j - 1] * b[id - 1] + Ddn[j * n + j] * bb;
                        }
                    }
                    if (i == 0 && yp > tol) {
                        dFeta = Dup[i * n + 0] * (g * h) + Dup[i * n + 1] * (g * H[id + n]);
                        dBeta = Dup[i * n + 0] * bb + Dup[i * n + 1] * b[id + n];
                    }
                    if (i == n - 1 && ym > tol) {
                        dFeta = Ddn[i * n + n - 2] * (g * H[id - n]) + Ddn[i * n + n - 1] * (g * h);
                        dBeta = Ddn[i * n + n - 2] * b[id - n] + Ddn[i * n + n - 1] * bb;
                    }
                    if (i > 0 && i < n - 1) {
                        if (yp > tol && ym > tol) {
                            dFeta = Dc[i * n + i - 1] * (g * H[id - n]) + Dc[i * n + i + 1] * (g * H[id + n]);
                            dBeta = Dc[i * n + i - 1] * b[id - n] + Dc[i * n + i + 1] * b[id + n];
                        } else if (yp > tol) {
                            dFeta = Dup[i * n + i] * (g * h) + Dup[i * n + i + 1] * (g * H[id + n]);
                            dBeta = Dup[i * n + i] * bb + Dup[i * n + i + 1] * b[id + n];
                        } else if (ym > tol) {
                            dFeta = Ddn[i * n + i - 1] * (g * H[id - n]) + Ddn[i * n + i] * (g * h);
                            dBeta = Ddn[i * n + i - 1] * b[id - n] + Ddn[i * n + i] * bb;
                        }
                    }
                }
                /* g/2 h^2 at the element's edges */
                const double pBD = c->half_g * h * h;
                double bxi = 0.0, beta = 0.0;
                if (j == 0) bxi += c->geomFace * pBD;
                if (j == n - 1) bxi += -c->geomFace * pBD;
                if (i == 0) beta += c->geomFace * pBD;
                if (i == n - 1) beta += -c->geomFace * pBD;
                const long x = (long)e * n2 + id;
                const double ye = Yeta[x], yx = Yxi[x], xe = Xeta[x], xx = Xxi[x], J = Jac[x];
                const double f2 = h * (ye * dFxi - yx * dFeta) + (ye * bxi - yx * beta);
                const double f3 = h * (-xe * dFxi + xx * dFeta) + (-xe * bxi + xx * beta);
                const double bx = ye * dBxi - yx * dBeta, by = -xe * dBxi + xx * dBeta;
                const long q = (long)e * n2 * NEQ + id;
                Qt[q + n2] = -J * f2 - g * J * h * bx;
                Qt[q + 2 * n2] = -J * f3 - g * J * h * by;
            }
    }
}

/* Analysis outputs after a step, with the new time t (called after t += dt
 * at src/deviceclass.cpp:1130-1141): okl/Analysis/ArrivalTimes.okl:16-62
 * (first t at which |h + b - h_zero| exceeds 5e-5 while the entry is still
 * the sentinel 1000.0) and okl/Analysis/MaximumElevation.okl:16-55 (running
 * std::max of h + b - h_zero). */
static void analysis(int K, int n2, double t, double h_zero, const double* Q, const double* B, double* AT,
                     double* ME) {
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e)
        for (int id = 0; id < n2; ++id) {
            const long x = (long)e * n2 + id;
            const double h = Q[(long)e * n2 * NEQ + id];
            if (AT && AT[x] == 1000.0 && fabs((h + B[x]) - h_zero) > 0.00005) AT[x] = t;
            if (ME) {
                const double fs = h + B[x] - h_zero;
                ME[x] = ME[x] < fs ? fs : ME[x];
            }
        }
}

/* ========================================================================= */
/* Public entry points                                                        */
/* ========================================================================= */

typedef struct {
    /* geometry and tables (borrowed) */
    const double *Jinv, *Yxi, *Yeta, *Xxi, *Xeta, *Bx, *By, *B, *nx, *ny, *scal;
    const double *D, *Dstrong, *Dhat, *VdmInv, *GLw, *EleSizes;
    const int *EdgeData, *EdgeReversed, *ElemToEdge, *MasterSlave, *Orientation;
    /* partial-dry treatment (PD = 1): difference matrices (src/basis.cpp:190-229) */
    const double *DcFD, *DfFD, *DbFD;
    int PD;
    /* Testcase 1 (manufactured solution): nodal coordinates */
    const double *X, *Y;
    int Testcase;
    /* analysis outputs updated after every step of oracle_timeloop (NULL:
     * off; the caller fills them with 1000.0 and 0) and the still-water
     * level they are measured from */
    double *ArrivalTimes, *MaxElevation;
    double h0;
} oracle_geom;

/* One right-hand-side evaluation Qt = L(q) (no AV), as the stage body of
 * src/deviceclass.cpp:957-1011 computes it. */
void oracle_rhs(int N, int K, int F, double g, double PosPresTOL, int ES, int NumFlux, const oracle_geom* G,
                const double* q, double* Qt, double* SurfaceParts_out) {
    const int ngl = N + 1;
    oconst c;
    fill_const(&c, ngl, g, (double)(N * (N + 1)) / 2.0, PosPresTOL, ES, 0, 0, 0);
    /* geomFace = 1/w_0 (main.cpp:921); w_0 = 2/(N(N+1)) exactly as computed by the basis */
    c.geomFace = 1.0 / (2.0 / (N * (N + 1.0)));
    const long nf = (long)F * ngl;
    double* qL = (double*)calloc(nf * NEQ, sizeof(double));
    double* qR = (double*)calloc(nf * NEQ, sizeof(double));
    double* bL = (double*)calloc(nf, sizeof(double));
    double* bR = (double*)calloc(nf, sizeof(double));
    double* SP = SurfaceParts_out ? SurfaceParts_out : (double*)calloc(nf * NEQ, sizeof(double));
    oracle_collect_bottom(F, ngl, G->EdgeData, G->B, bL, bR);
    if (G->Testcase == 1)
        collect_edge_conv(F, ngl, G->EdgeData, q, G->X, G->Y, bL, bR, 0.0, qL, qR);
    else
        oracle_collect_edge_walls(F, ngl, G->EdgeData, q, G->nx, G->ny, qL, qR);
    volume_fluxdiff(&c, K, G->Jinv, G->Yxi, G->Yeta, G->Xxi, G->Xeta, q, G->D, G->Bx, G->By, Qt);
    if (G->PD) {
        int* dry = (int*)calloc(K, sizeof(int));
        find_dry(&c, K, q, dry);
        volume_partial_dry(&c, K, G->Jinv, G->Yxi, G->Yeta, G->Xxi, G->Xeta, q, dry, G->DcFD, G->DfFD, G->DbFD,
                           G->B, Qt);
        free(dry);
    }
    num_fluxes(&c, NumFlux, F, G->EdgeReversed, G->nx, G->ny, G->scal, qL, qR, bL, bR, SP);
    surface_lift(ngl, K, G->Jinv, G->MasterSlave, G->Orientation, G->ElemToEdge, SP, Qt);
    if (G->Testcase == 1) add_conv_source(&c, K, G->Bx, G->By, G->B, G->X, G->Y, 0.0, Qt);
    free(qL); free(qR); free(bL); free(bR);
    if (!SurfaceParts_out) free(SP);
}

/* Per-element shock-capturing viscosity (for tests of that kernel alone). */
void oracle_shock_capturing(int N, int K, double eps0, double sigmaMin, double sigmaMax, const double* q,
                            const double* b, const double* VdmInv, double* ViscPara) {
    oconst c;
    fill_const(&c, N + 1, 9.81, 1.0, 0.0, 1, eps0, sigmaMin, sigmaMax);
    shock_capturing(&c, K, q, b, VdmInv, ViscPara);
}

/* The time loop of src/deviceclass.cpp:630-1335 for the SolidWalls/periodic
 * edge gather, flux-differencing volume term, ES Riemann solver NumFlux in
 * {0,2,3}, low-storage (rkSSP=0) or SSP (rkSSP=1) RK, optional artificial
 * viscosity (AV) and positivity limiter (PP).  Runs while t<T and, when
 * max_steps>0, at most max_steps steps.  q is advanced in place.
 * dt_log (optional, length max_steps) receives each step's dt.            */
int oracle_timeloop(int N, int K, int F, const oracle_geom* G, double* q, double g, double PosPresTOL, int ES,
                    int NumFlux, int rkStages, const double* rkA, const double* rkB, const double* rkC, int rkSSP,
                    int AV, int PP, double eps0, double sigmaMin, double sigmaMax, double minEleSize, double CFL,
                    double DFL, double T, int max_steps, double* t_out, int* steps_out, double* dt_log,
                    double* visc_out) {
    const int ngl = N + 1, n2 = ngl * ngl;
    oconst c;
    fill_const(&c, ngl, g, 0.0, PosPresTOL, ES, eps0, sigmaMin, sigmaMax);
    c.geomFace = 1.0 / (2.0 / (N * (N + 1.0)));
    const long nd = (long)K * n2 * NEQ, nf = (long)F * ngl;
    double* Qt = (double*)calloc(nd, sizeof(double));
    double* gRK = (double*)calloc(nd, sizeof(double));
    double* Qtmp = rkSSP ? (double*)calloc(nd, sizeof(double)) : NULL;
    double* qL = (double*)calloc(nf * NEQ, sizeof(double));
    double* qR = (double*)calloc(nf * NEQ, sizeof(double));
    double* bL = (double*)calloc(nf, sizeof(double));
    double* bR = (double*)calloc(nf, sizeof(double));
    double* SP = (double*)calloc(nf * NEQ, sizeof(double));
    int* dry = G->PD ? (int*)calloc(K, sizeof(int)) : NULL;
    double *VP = NULL, *GX = NULL, *GY = NULL, *SGX = NULL, *SGY = NULL, *VPL = NULL, *VPR = NULL;
    double *GXL = NULL, *GXR = NULL, *GYL = NULL, *GYR = NULL, *SPV = NULL;
    if (AV) {
        VP = (double*)calloc(K, sizeof(double));
        GX = (double*)calloc((long)K * n2 * 2, sizeof(double));
        GY = (double*)calloc((long)K * n2 * 2, sizeof(double));
        SGX = (double*)calloc(nf * 2, sizeof(double));
        SGY = (double*)calloc(nf * 2, sizeof(double));
        VPL = (double*)calloc(F, sizeof(double));
        VPR = (double*)calloc(F, sizeof(double));
        GXL = (double*)calloc(nf * 2, sizeof(double));
        GXR = (double*)calloc(nf * 2, sizeof(double));
        GYL = (double*)calloc(nf * 2, sizeof(double));
        GYR = (double*)calloc(nf * 2, sizeof(double));
        SPV = (double*)calloc(nf * 2, sizeof(double));
    }
    oracle_collect_bottom(F, ngl, G->EdgeData, G->B, bL, bR);
    double t = 0.0;
    int steps = 0;
    while (t < T && (max_steps <= 0 || steps < max_steps)) {
        const double lam = lambda_max(&c, K, q);
        const double dt_i = minEleSize / (ngl)*CFL / lam;
        double dt;
        if (AV) {
            shock_capturing(&c, K, q, G->B, G->VdmInv, VP);
            double vmax = 0.0;
            for (int e = 0; e < K; ++e) vmax = fmax(vmax, VP[e]);
            const double dt_v = DFL / (pow(ngl, 2)) * pow(minEleSize, 2) / vmax;
            dt = fmin(T - t, fmin(dt_i, dt_v));
        } else {
            dt = fmin(T - t, dt_i);
        }
        if (dt_log) dt_log[steps] = dt;
        if (rkSSP) memcpy(Qtmp, q, nd * sizeof(double));
        for (int s = 0; s < rkStages; ++s) {
            /* stage time (src/deviceclass.cpp:944-952) */
            static const double rkD[3] = {0.0, 1.0, 0.5};
            double ts = t;
            ts += (rkSSP ? rkD[s < 3 ? s : 0] : rkB[s]) * dt;
            if (G->Testcase == 1)
                collect_edge_conv(F, ngl, G->EdgeData, q, G->X, G->Y, bL, bR, ts, qL, qR);
            else
                oracle_collect_edge_walls(F, ngl, G->EdgeData, q, G->nx, G->ny, qL, qR);
            volume_fluxdiff(&c, K, G->Jinv, G->Yxi, G->Yeta, G->Xxi, G->Xeta, q, G->D, G->Bx, G->By, Qt);
            if (G->PD) {
                find_dry(&c, K, q, dry);
                volume_partial_dry(&c, K, G->Jinv, G->Yxi, G->Yeta, G->Xxi, G->Xeta, q, dry, G->DcFD, G->DfFD,
                                   G->DbFD, G->B, Qt);
            }
            num_fluxes(&c, NumFlux, F, G->EdgeReversed, G->nx, G->ny, G->scal, qL, qR, bL, bR, SP);
            surface_lift(ngl, K, G->Jinv, G->MasterSlave, G->Orientation, G->ElemToEdge, SP, Qt);
            if (AV) {
                if (s > 0) shock_capturing(&c, K, q, G->B, G->VdmInv, VP);
                num_fluxes_gradient(&c, F, G->EdgeData, G->nx, G->ny, G->scal, qL, qR, SGX, SGY);
                calc_gradient(&c, K, G->Jinv, G->Yxi, G->Yeta, G->Xxi, G->Xeta, q, G->Dhat, GX, GY);
                surface_lift_grad(ngl, K, G->Jinv, G->MasterSlave, G->Orientation, G->ElemToEdge, SGX, SGY, GX, GY);
                scale_gradient(ngl, K, q, GX, GY);
                collect_edge_gradient(ngl, F, G->EdgeData, GX, GY, VP, VPL, VPR, GXL, GXR, GYL, GYR);
                volume_viscous(&c, K, G->Jinv, G->Yxi, G->Yeta, G->Xxi, G->Xeta, GX, GY, G->Dstrong, VP, Qt);
                num_fluxes_viscous(&c, F, G->EdgeData, G->nx, G->ny, G->scal, VPL, VPR, GXL, GXR, GYL, GYR, SPV);
                surface_lift_visc(ngl, K, G->Jinv, G->MasterSlave, G->Orientation, G->ElemToEdge, SPV, Qt);
            }
            if (G->Testcase == 1) add_conv_source(&c, K, G->Bx, G->By, G->B, G->X, G->Y, ts, Qt);
            if (rkSSP) {
                const double A = rkA[s], Bc = rkB[s], C = rkC[s];
#pragma omp parallel for schedule(static)
                for (long id = 0; id < nd; ++id) q[id] = A * Qtmp[id] + Bc * q[id] + C * dt * Qt[id];
            } else {
                const double A = rkA[s], C = rkC[s];
#pragma omp parallel for schedule(static)
                for (long id = 0; id < nd; ++id) {
                    gRK[id] = A * gRK[id] + Qt[id];
                    q[id] += C * dt * gRK[id];
                }
            }
            if (PP) pos_pres(&c, K, G->EleSizes, G->GLw, G->Jinv, q);
        }
        t += dt;
        ++steps;
        if (G->ArrivalTimes || G->MaxElevation)
            analysis(K, n2, t, G->h0, q, G->B, G->ArrivalTimes, G->MaxElevation);
    }
    if (visc_out && AV) memcpy(visc_out, VP, (size_t)K * sizeof(double));
    if (t_out) *t_out = t;
    if (steps_out) *steps_out = steps;
    free(Qt); free(gRK); free(Qtmp); free(qL); free(qR); free(bL); free(bR); free(SP);
    free(VP); free(GX); free(GY); free(SGX); free(SGY); free(VPL); free(VPR);
    free(GXL); free(GXR); free(GYL); free(GYR); free(SPV); free(dry);
    return 0;
}

/* Stand-alone kernels for per-kernel parity tests. */
void oracle_lambda_max(int N, int K, double g, double PosPresTOL, const double* q, double* out) {
    oconst c;
    fill_const(&c, N + 1, g, 1.0, PosPresTOL, 1, 0, 0, 0);
    *out = lambda_max(&c, K, q);
}

void oracle_pos_pres(int N, int K, double PosPresTOL, const double* EleSizes, const double* GLw, const double* Jinv,
                     double* q) {
    oconst c;
    fill_const(&c, N + 1, 9.81, 1.0, PosPresTOL, 1, 0, 0, 0);
    pos_pres(&c, K, EleSizes, GLw, Jinv, q);
}

/* Viscous right-hand side contribution (AV chain of one stage) added to Qt:
 * src/deviceclass.cpp:1038-1094.  ViscPara must hold the element viscosity. */
void oracle_viscous_rhs(int N, int K, int F, const oracle_geom* G, double PosPresTOL, const double* q,
                        const double* ViscPara, double* Qt) {
    const int ngl = N + 1, n2 = ngl * ngl;
    oconst c;
    fill_const(&c, ngl, 9.81, 0.0, PosPresTOL, 1, 0, 0, 0);
    c.geomFace = 1.0 / (2.0 / (N * (N + 1.0)));
    const long nf = (long)F * ngl;
    double* qL = (double*)calloc(nf * NEQ, sizeof(double));
    double* qR = (double*)calloc(nf * NEQ, sizeof(double));
    double* GX = (double*)calloc((long)K * n2 * 2, sizeof(double));
    double* GY = (double*)calloc((long)K * n2 * 2, sizeof(double));
    double* SGX = (double*)calloc(nf * 2, sizeof(double));
    double* SGY = (double*)calloc(nf * 2, sizeof(double));
    double* VPL = (double*)calloc(F, sizeof(double));
    double* VPR = (double*)calloc(F, sizeof(double));
    double* GXL = (double*)calloc(nf * 2, sizeof(double));
    double* GXR = (double*)calloc(nf * 2, sizeof(double));
    double* GYL = (double*)calloc(nf * 2, sizeof(double));
    double* GYR = (double*)calloc(nf * 2, sizeof(double));
    double* SPV = (double*)calloc(nf * 2, sizeof(double));
    oracle_collect_edge_walls(F, ngl, G->EdgeData, q, G->nx, G->ny, qL, qR);
    num_fluxes_gradient(&c, F, G->EdgeData, G->nx, G->ny, G->scal, qL, qR, SGX, SGY);
    calc_gradient(&c, K, G->Jinv, G->Yxi, G->Yeta, G->Xxi, G->Xeta, q, G->Dhat, GX, GY);
    surface_lift_grad(ngl, K, G->Jinv, G->MasterSlave, G->Orientation, G->ElemToEdge, SGX, SGY, GX, GY);
    scale_gradient(ngl, K, q, GX, GY);
    collect_edge_gradient(ngl, F, G->EdgeData, GX, GY, ViscPara, VPL, VPR, GXL, GXR, GYL, GYR);
    volume_viscous(&c, K, G->Jinv, G->Yxi, G->Yeta, G->Xxi, G->Xeta, GX, GY, G->Dstrong, ViscPara, Qt);
    num_fluxes_viscous(&c, F, G->EdgeData, G->nx, G->ny, G->scal, VPL, VPR, GXL, GXR, GYL, GYR, SPV);
    surface_lift_visc(ngl, K, G->Jinv, G->MasterSlave, G->Orientation, G->ElemToEdge, SPV, Qt);
    free(qL); free(qR); free(GX); free(GY); free(SGX); free(SGY); free(VPL); free(VPR);
    free(GXL); free(GXR); free(GYL); free(GYR); free(SPV);
}
