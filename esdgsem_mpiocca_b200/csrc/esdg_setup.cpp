// Host-side set-up for the ES-DGSEM shallow-water engine: LGL basis and
// operators, Cartesian / mapped / ISM-V2 meshes, curvilinear geometry,
// face and element connectivity tables, split-form bathymetry gradient and
// the quadrature diagnostics.  Everything here runs once per problem on the
// host; the per-step work lives in esdg_kernels.cu.
//
// Each routine states the reference routine whose numbers it reproduces.
// Paths are relative to the ESDGSEM_MPIOCCA source tree.

#include "esdg_setup.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <algorithm>

namespace esdg {

// ---------------------------------------------------------------------------
// Legendre polynomials and quadrature (Kopriva, "Implementing Spectral
// Methods for PDEs", algorithms 22-25).  Same Newton start values, iteration
// cap and stopping test as src/basis.cpp:593-788 so that nodes agree to the
// last bit.
// ---------------------------------------------------------------------------

static void legendre_L_dL(int n, double x, double* L, double* dL) {
    // src/basis.cpp:564-610 (three-term recursion for L_n and L_n').
    if (n == 0) { *L = 1.0; *dL = 0.0; return; }
    if (n == 1) { *L = x; *dL = 1.0; return; }
    double Lm2 = 1.0, Lm1 = x, dLm2 = 0.0, dLm1 = 1.0;
    double Lk = 0.0, dLk = 0.0;
    for (int k = 2; k <= n; ++k) {
        Lk = ((2.0 * k - 1.0) / k) * x * Lm1 - (k - 1.0) / k * Lm2;
        dLk = dLm2 + (2.0 * k - 1.0) * Lm1;
        Lm2 = Lm1; Lm1 = Lk; dLm2 = dLm1; dLm1 = dLk;
    }
    *L = Lk; *dL = dLk;
}

static void lobatto_q(int N, double x, double* q, double* dq, double* LN) {
    // q(x) = L_{N+1} - L_{N-1} and q'(x); src/basis.cpp:628-658.
    double Lm2 = 1.0, Lm1 = x, dLm2 = 0.0, dLm1 = 1.0, dL = 0.0;
    double L = 0.0;
    for (int k = 2; k <= N; ++k) {
        L = (2.0 * k - 1.0) / k * x * Lm1 - (k - 1.0) / k * Lm2;
        dL = dLm2 + (2.0 * k - 1.0) * Lm1;
        if (k < N) { Lm2 = Lm1; Lm1 = L; dLm2 = dLm1; dLm1 = dL; }
    }
    const int k = N + 1;
    const double Lp1 = (2.0 * k - 1.0) / k * x * L - (k - 1.0) / k * Lm1;
    const double dLp1 = dLm1 + (2.0 * k - 1.0) * L;
    *q = Lp1 - Lm1;
    *dq = dLp1 - dLm1;
    *LN = L;
}

void lgl_nodes_weights(int N, double* x, double* w) {
    // src/basis.cpp:662-730.
    const int ngl = N + 1;
    const int newton_it = 4;
    const double TOL = 4. * std::pow(10., -16);
    double q = 0, dq = 0, LN = 0;
    if (N == 1) {
        x[0] = -1.0; w[0] = 1.0; x[1] = 1.0; w[1] = 1.0;
        return;
    }
    x[0] = -1.0;
    w[0] = 2.0 / (N * (N + 1.0));
    x[ngl - 1] = 1.0;
    w[ngl - 1] = w[0];
    if (N == 2) {
        lobatto_q(N, 0.0, &q, &dq, &LN);
        x[1] = 0.0;
        w[1] = 2.0 / ((double)(N * (N + 1)) * (LN * LN));
        return;
    }
    for (int j = 1; j <= (int)std::floor(N / 2.0); ++j) {
        x[j] = -std::cos((j + 1.0 / 4.0) * M_PI / N - 3.0 / (8.0 * N * M_PI) * 1.0 / (j + 1.0 / 4.0));
        for (int k = 0; k <= newton_it; ++k) {
            lobatto_q(N, x[j], &q, &dq, &LN);
            const double delta = -q / dq;
            x[j] = x[j] + delta;
            if (std::fabs(delta) <= TOL * std::fabs(x[j])) break;
        }
        lobatto_q(N, x[j], &q, &dq, &LN);
        x[ngl - j - 1] = -x[j];
        w[j] = 2.0 / ((double)(N * (N + 1)) * (LN * LN));
        w[ngl - j - 1] = w[j];
    }
    if (N % 2 == 0) {
        lobatto_q(N, 0.0, &q, &dq, &LN);
        x[N / 2] = 0.0;
        w[N / 2] = 2.0 / ((double)(N * (N + 1)) * (LN * LN));
    }
}

void gauss_nodes_weights(int N, double* x, double* w) {
    // src/basis.cpp:733-788 (N+1 Gauss-Legendre points).
    const int ngl = N + 1;
    const int newton_it = 4;
    const double TOL = 4. * std::pow(10., -16);
    double L1 = 0, L2 = 0;
    if (N == 0) { x[0] = 0.0; w[0] = 2.0; return; }
    if (N == 1) {
        x[0] = -std::sqrt(1.0 / 3.0); w[0] = 1.0; x[1] = -x[0]; w[1] = w[0];
        return;
    }
    for (int j = 0; j < (int)std::floor((N + 1.0) / 2.0); ++j) {
        x[j] = -std::cos((2.0 * j + 1.0) / (2.0 * N + 2.0) * M_PI);
        for (int k = 0; k <= newton_it; ++k) {
            legendre_L_dL(N + 1, x[j], &L1, &L2);
            const double delta = -L1 / L2;
            x[j] = x[j] + delta;
            if (std::fabs(delta) <= TOL * std::fabs(x[j])) break;
        }
        legendre_L_dL(N + 1, x[j], &L1, &L2);
        x[ngl - j - 1] = -x[j];
        w[j] = 2.0 / ((1.0 - x[j] * x[j]) * (L2 * L2));
        w[ngl - j - 1] = w[j];
    }
    if (N % 2 == 0) {
        legendre_L_dL(N + 1, 0.0, &L1, &L2);
        x[N / 2] = 0.0;
        w[N / 2] = 2.0 / (L2 * L2);
    }
}

static void barycentric_weights(int n, const double* x, double* wb) {
    // src/basis.cpp:825-849, src/Mesh.cpp:1832-1858 and :1989-2013.
    for (int i = 0; i < n; ++i) wb[i] = 1.0;
    for (int j = 1; j < n; ++j)
        for (int k = 0; k < j; ++k) {
            wb[k] = wb[k] * (x[k] - x[j]);
            wb[j] = wb[j] * (x[j] - x[k]);
        }
    for (int j = 0; j < n; ++j) wb[j] = 1.0 / wb[j];
}

static void lagrange_basis_at(double x0, int n, const double* x, const double* wb, double* P) {
    // src/basis.cpp:791-822.
    bool match = false;
    const double TOL = 4. * std::pow(10., -16);
    for (int j = 0; j < n; ++j) {
        P[j] = 0.0;
        if (std::fabs(x0 - x[j]) < TOL) { match = true; P[j] = 1; }
    }
    if (!match) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) {
            const double t = wb[j] / (x0 - x[j]);
            P[j] = t;
            s = s + t;
        }
        for (int j = 0; j < n; ++j) P[j] = P[j] / s;
    }
}

void build_basis(int N, int flux_differencing, Basis* B) {
    // src/basis.cpp:28-188 (constructor) and :495-561 (ModalTrafoMatrix).
    const int n = N + 1, n2 = n * n;
    B->N = N;
    B->ngl = n;
    B->xGL.assign(n, 0.0); B->wGL.assign(n, 0.0);
    B->xG.assign(n, 0.0);  B->wG.assign(n, 0.0);
    B->wbary.assign(n, 0.0);
    B->D0.assign(n2, 0.0); B->D.assign(n2, 0.0); B->Dstrong.assign(n2, 0.0);
    B->Dhat.assign(n2, 0.0); B->VdmInv.assign(n2, 0.0);
    lgl_nodes_weights(N, B->xGL.data(), B->wGL.data());
    gauss_nodes_weights(N, B->xG.data(), B->wG.data());
    barycentric_weights(n, B->xGL.data(), B->wbary.data());
    // Collocation derivative matrix (Kopriva algorithm 37); the diagonal is
    // the negative row sum accumulated in column order.
    std::vector<double> Dm(n2, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (i != j) {
                const int id = i * n + j;
                Dm[id] = (B->wbary[j] / B->wbary[i]) * (1.0 / (B->xGL[i] - B->xGL[j]));
                Dm[i * n + i] = Dm[i * n + i] - Dm[id];
            }
    for (int id = 0; id < n2; ++id) {
        B->D0[id] = Dm[id];
        B->Dstrong[id] = Dm[id];
        B->D[id] = flux_differencing ? 2.0 * Dm[id] : Dm[id];
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            B->Dhat[i * n + j] = -B->wGL[j] * B->D0[j * n + i] / B->wGL[i];
    B->D[0] = B->D[0] + 1.0 / B->wGL[0];
    B->D[n2 - 1] = B->D[n2 - 1] - 1.0 / B->wGL[n - 1];
    B->Dstrong[0] = B->D0[0] + 1.0 / B->wGL[0];
    B->Dstrong[n2 - 1] = B->D0[n2 - 1] - 1.0 / B->wGL[n - 1];
    // Nodal -> orthonormal-Legendre modal transform through Gauss quadrature.
    std::vector<double> Vtmp(n2, 0.0), Itmp(n2, 0.0), P(n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double L, dL;
            legendre_L_dL(j, B->xG[i], &L, &dL);
            Vtmp[j * n + i] = L * std::sqrt(j + 0.5) * B->wG[i];
        }
    for (int i = 0; i < n; ++i) {
        lagrange_basis_at(B->xG[i], n, B->xGL.data(), B->wbary.data(), P.data());
        for (int j = 0; j < n; ++j) Itmp[i * n + j] = P[j];
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int l = 0; l < n; ++l)
                B->VdmInv[i * n + j] += Vtmp[i * n + l] * Itmp[l * n + j];
}

// ---------------------------------------------------------------------------
// Mesh and geometry.
// ---------------------------------------------------------------------------

Mesh::Mesh(int N_) : N(N_), ngl(N_ + 1) { build_basis(N_, 1, &basis); }

void Mesh::alloc(int K_, int F_) {
    K = K_; F = F_;
    const size_t nn = (size_t)K * ngl * ngl;
    x.assign(nn, 0.0); y.assign(nn, 0.0);
    xXi.assign(nn, 0.0); xEta.assign(nn, 0.0); yXi.assign(nn, 0.0); yEta.assign(nn, 0.0);
    J.assign(nn, 0.0);
    nxSide.assign((size_t)K * 4 * ngl, 0.0);
    nySide.assign((size_t)K * 4 * ngl, 0.0);
    scalSide.assign((size_t)K * 4 * ngl, 0.0);
    EdgeInfo.assign((size_t)F * 7, 0);
    ElementToEdge.assign((size_t)K * 4, 0);
}

void curve_nodes_weights(int m, double* xc, double* wb) {
    for (int k = 0; k <= m; ++k) xc[k] = -std::cos(k * M_PI / m);
    barycentric_weights(m + 1, xc, wb);
}

// Curve evaluation on Chebyshev-Gauss-Lobatto samples: src/Mesh.cpp:1861-1987.
struct Curve {
    int m = 0;                         // polynomial order of the boundary curves
    std::vector<double> xc, wb;        // nodes -cos(k pi/m) and barycentric weights
    void init(int order) {
        m = order;
        xc.resize(m + 1); wb.resize(m + 1);
        for (int k = 0; k <= m; ++k) xc[k] = -std::cos(k * M_PI / m);
        barycentric_weights(m + 1, xc.data(), wb.data());
    }
    double eval(const double* f, double s) const {
        double num = 0.0, den = 0.0, out = 0.0;
        bool at = false;
        for (int j = 0; j <= m; ++j)
            if (std::fabs(s - xc[j]) < std::pow(10.0, -12)) { at = true; out = f[j]; }
        if (!at) {
            for (int j = 0; j <= m; ++j) {
                const double t = wb[j] / (s - xc[j]);
                num += t * f[j];
                den += t;
            }
            out = num / den;
        }
        return out;
    }
};

static double transfinite(const Curve& C, const double* G1, const double* G2, const double* G3,
                          const double* G4, double psi, double eta) {
    // src/Mesh.cpp:1619-1640.
    const double x1r = C.eval(G1, -1.0), x2r = C.eval(G1, 1.0);
    const double x3r = C.eval(G3, 1.0), x4r = C.eval(G3, -1.0);
    const double x1 = C.eval(G1, psi), x2 = C.eval(G2, eta);
    const double x3 = C.eval(G3, psi), x4 = C.eval(G4, eta);
    return 0.5 * ((1.0 - psi) * x4 + (1.0 + psi) * x2 + (1.0 - eta) * x1 + (1.0 + eta) * x3) -
           0.25 * ((1.0 - psi) * ((1.0 - eta) * x1r + (1.0 + eta) * x4r) +
                   (1.0 + psi) * ((1.0 - eta) * x2r + (1.0 + eta) * x3r));
}

static double bilinear(const double* c, double psi, double eta) {
    // src/Mesh.cpp:1642-1650.
    return 0.25 * (c[0] * (1.0 - psi) * (1.0 - eta) + c[1] * (1.0 + psi) * (1.0 - eta) +
                   c[2] * (1.0 + psi) * (1.0 + eta) + c[3] * (1.0 - psi) * (1.0 + eta));
}

// Metric terms, Jacobian and outward side normals of one element from its
// nodal coordinates (src/Mesh.cpp:1667-1808: collocation derivatives of the
// interpolated map, so the discrete metric identities hold exactly in 2-D).
void Mesh::element_geometry(int e, const double* xp, const double* yp) {
    const int n = ngl, n2 = n * n;
    const double* D = basis.D0.data();
    double* ex = &x[(size_t)e * n2];   double* ey = &y[(size_t)e * n2];
    double* xx = &xXi[(size_t)e * n2]; double* xe = &xEta[(size_t)e * n2];
    double* yx = &yXi[(size_t)e * n2]; double* ye = &yEta[(size_t)e * n2];
    double* Je = &J[(size_t)e * n2];
    for (int id = 0; id < n2; ++id) { ex[id] = xp[id]; ey[id] = yp[id]; }
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int ij = j * n + i;
            double a = 0, b = 0, c = 0, d = 0;
            for (int k = 0; k < n; ++k) {
                a += D[i * n + k] * xp[j * n + k];
                b += D[j * n + k] * xp[k * n + i];
                c += D[i * n + k] * yp[j * n + k];
                d += D[j * n + k] * yp[k * n + i];
            }
            xx[ij] = a; xe[ij] = b; yx[ij] = c; ye[ij] = d;
            Je[ij] = a * d - b * c;
        }
    double* nx = &nxSide[(size_t)e * 4 * n];
    double* ny = &nySide[(size_t)e * 4 * n];
    double* sc = &scalSide[(size_t)e * 4 * n];
    for (int j = 0; j < n; ++j) {
        const int s2 = n + j, s4 = 3 * n + j;
        const int Nj = j * n + n - 1, Zj = j * n;
        double yE = ye[Nj], xE = xe[Nj], Jt = Je[Nj];
        sc[s2] = std::sqrt(yE * yE + xE * xE);
        nx[s2] = std::copysign(1.0, Jt) * (yE / sc[s2]);
        ny[s2] = std::copysign(1.0, Jt) * (-xE / sc[s2]);
        yE = ye[Zj]; xE = xe[Zj]; Jt = Je[Zj];
        sc[s4] = std::sqrt(yE * yE + xE * xE);
        nx[s4] = -std::copysign(1.0, Jt) * (yE / sc[s4]);
        ny[s4] = -std::copysign(1.0, Jt) * (-xE / sc[s4]);
    }
    for (int i = 0; i < n; ++i) {
        const int s1 = i, s3 = 2 * n + i;
        const int iZ = i, iN = (n - 1) * n + i;
        double yX = yx[iZ], xX = xx[iZ], Jt = Je[iZ];
        sc[s1] = std::sqrt(yX * yX + xX * xX);
        nx[s1] = -std::copysign(1.0, Jt) * (-yX / sc[s1]);
        ny[s1] = -std::copysign(1.0, Jt) * (xX / sc[s1]);
        yX = yx[iN]; xX = xx[iN]; Jt = Je[iN];
        sc[s3] = std::sqrt(yX * yX + xX * xX);
        nx[s3] = std::copysign(1.0, Jt) * (-yX / sc[s3]);
        ny[s3] = std::copysign(1.0, Jt) * (xX / sc[s3]);
    }
}

void Mesh::finish_tables() {
    // Per-side master/slave flags and orientations (src/Mesh.cpp:87-111),
    // face-wise normals taken from the left element (src/Mesh.cpp:281-305).
    const int n = ngl;
    MasterSlave.assign((size_t)K * 4, 0);
    Orientation.assign((size_t)K * 4, 0);
    for (int e = 0; e < K; ++e)
        for (int s = 0; s < 4; ++s) {
            const int id = e * 4 + s;
            const int f = ElementToEdge[id] - 1;
            if (f < 0 || f >= F) throw std::runtime_error("element side without a face");
            if (EdgeInfo[(size_t)f * 7 + 2] == e) { MasterSlave[id] = 1; Orientation[id] = 1; }
            else { MasterSlave[id] = -1; Orientation[id] = EdgeInfo[(size_t)f * 7 + 6]; }
        }
    nxFace.assign((size_t)F * n, 0.0);
    nyFace.assign((size_t)F * n, 0.0);
    scalFace.assign((size_t)F * n, 0.0);
    for (int f = 0; f < F; ++f)
        for (int i = 0; i < n; ++i) {
            const size_t loc = (size_t)EdgeInfo[(size_t)f * 7 + 2] * 4 * n + EdgeInfo[(size_t)f * 7 + 4] * n + i;
            nxFace[(size_t)f * n + i] = nxSide[loc];
            nyFace[(size_t)f * n + i] = nySide[loc];
            scalFace[(size_t)f * n + i] = scalSide[loc];
        }
}

// Uniform Cartesian grid with optional periodic wrap, numbered as
// src/Mesh.cpp:316-696: horizontal faces first (row by row), then vertical
// faces; the flag named periodic_y wraps the horizontal faces (bottom to top).
void Mesh::generate_cartesian(double xL, double xR, double yL, double yR, int NX, int NY,
                              bool periodic_wrap_rows, bool periodic_wrap_cols) {
    const int n = ngl, n2 = n * n;
    int Fc = (NX + 1) * NY + (NY + 1) * NX;
    if (periodic_wrap_rows) Fc -= NX;
    if (periodic_wrap_cols) Fc -= NY;
    alloc(NX * NY, Fc);
    has_bottom = false;
    const double dX = (xR - xL) / NX, dY = (yR - yL) / NY;
    const double x_xi = 0.5 * dX, y_eta = 0.5 * dY, Jac = x_xi * y_eta;
    const double* xg = basis.xGL.data();
    for (int ieY = 0; ieY < NY; ++ieY)
        for (int ieX = 0; ieX < NX; ++ieX)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    const size_t id = (size_t)(ieY * NX + ieX) * n2 + j * n + i;
                    x[id] = xL + (xg[i] + 1.0) / 2.0 * dX + ieX * dX;
                    y[id] = yL + (xg[j] + 1.0) / 2.0 * dY + ieY * dY;
                }
    for (size_t id = 0; id < (size_t)K * n2; ++id) {
        xXi[id] = x_xi; xEta[id] = 0.0; yXi[id] = 0.0; yEta[id] = y_eta; J[id] = Jac;
    }
    auto set_side = [&](int e, int s, double nxv, double nyv, double sc) {
        for (int i = 0; i < n; ++i) {
            const size_t id = (size_t)e * 4 * n + s * n + i;
            nxSide[id] = nxv; nySide[id] = nyv; scalSide[id] = sc;
        }
    };
    auto finish_face = [&](int is) {
        int* E = &EdgeInfo[(size_t)(is - 1) * 7];
        E[0] = 0; E[1] = 0; E[6] = 1;
        ElementToEdge[E[2] * 4 + E[4]] = is;
        if (E[3] != -1) ElementToEdge[E[3] * 4 + E[5]] = is;
    };
    const int jLoop = periodic_wrap_rows ? NY - 1 : NY;
    for (int j = 0; j <= jLoop; ++j)
        for (int i = 0; i < NX; ++i) {
            const int is = j * NX + i + 1;
            int* E = &EdgeInfo[(size_t)(is - 1) * 7];
            if (j == 0) {
                E[2] = i; E[4] = 0; E[3] = -1; E[5] = -1;
                set_side(E[2], E[4], 0.0, -1.0, x_xi);
                if (periodic_wrap_rows) {
                    E[3] = (NY - 1) * NX + i; E[5] = 2;
                    set_side(E[3], E[5], 0.0, 1.0, x_xi);
                }
            } else if (j == NY) {
                E[2] = (NY - 1) * NX + i; E[4] = 2; E[3] = -1; E[5] = -1;
                set_side(E[2], E[4], 0.0, 1.0, x_xi);
            } else {
                E[2] = (j - 1) * NX + i; E[3] = j * NX + i; E[4] = 2; E[5] = 0;
                set_side(E[2], E[4], 0.0, 1.0, x_xi);
                set_side(E[3], E[5], 0.0, -1.0, x_xi);
            }
            finish_face(is);
        }
    const int iLoop = periodic_wrap_cols ? NX - 1 : NX;
    for (int j = 0; j < NY; ++j)
        for (int i = 0; i <= iLoop; ++i) {
            const int is = (jLoop + 1) * NX + (j * (iLoop + 1) + i) + 1;
            int* E = &EdgeInfo[(size_t)(is - 1) * 7];
            if (i == 0) {
                E[2] = j * NX; E[4] = 3; E[3] = -1; E[5] = -1;
                set_side(E[2], E[4], -1.0, 0.0, y_eta);
                if (periodic_wrap_cols) {
                    E[3] = (j + 1) * NX - 1; E[5] = 1;
                    set_side(E[3], E[5], 1.0, 0.0, y_eta);
                }
            } else if (i == NX) {
                E[2] = (j + 1) * NX - 1; E[4] = 1; E[3] = -1; E[5] = -1;
                set_side(E[2], E[4], 1.0, 0.0, y_eta);
            } else {
                E[2] = j * NX + i - 1; E[3] = j * NX + i; E[4] = 1; E[5] = 3;
                set_side(E[2], E[4], 1.0, 0.0, y_eta);
                set_side(E[3], E[5], -1.0, 0.0, y_eta);
            }
            finish_face(is);
        }
    finish_tables();
}

// One quadrilateral given by its corners (counter-clockwise) and, for curved
// sides, (m+1) Chebyshev-Lobatto samples per side; the straight sides are
// sampled from their corners (src/Mesh.cpp:1000-1081).  Geometry by the
// transfinite map when any side is curved, else bilinear.
void Mesh::element_from_curves(int e, const double* cx, const double* cy, const double* cb,
                               const double* const* gx, const double* const* gy,
                               const double* const* gb, const int* curved_side, int m) {
    const int n = ngl, n2 = n * n;
    Curve C;
    C.init(m);
    bool curved = false;
    for (int s = 0; s < 4; ++s) curved = curved || curved_side[s];
    std::vector<double> G[3][4];
    static const int ends[4][2] = {{0, 1}, {1, 2}, {3, 2}, {0, 3}};
    for (int s = 0; s < 4; ++s)
        for (int c = 0; c < 3; ++c) G[c][s].assign(m + 1, 0.0);
    for (int s = 0; s < 4; ++s) {
        if (curved_side[s]) {
            for (int k = 0; k <= m; ++k) {
                G[0][s][k] = gx[s][k];
                G[1][s][k] = gy[s][k];
                if (cb && gb) G[2][s][k] = gb[s][k];
            }
        } else {
            const int a = ends[s][0], b = ends[s][1];
            for (int k = 0; k <= m; ++k) {
                G[0][s][k] = ((cx[b] - cx[a]) * C.xc[k] + cx[a] + cx[b]) / 2.0;
                G[1][s][k] = ((cy[b] - cy[a]) * C.xc[k] + cy[a] + cy[b]) / 2.0;
                if (cb) G[2][s][k] = ((cb[b] - cb[a]) * C.xc[k] + cb[a] + cb[b]) / 2.0;
            }
        }
    }
    std::vector<double> xp(n2), yp(n2), bp(n2);
    const double* xg = basis.xGL.data();
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int ij = j * n + i;
            if (curved) {
                xp[ij] = transfinite(C, G[0][0].data(), G[0][1].data(), G[0][2].data(), G[0][3].data(), xg[i], xg[j]);
                yp[ij] = transfinite(C, G[1][0].data(), G[1][1].data(), G[1][2].data(), G[1][3].data(), xg[i], xg[j]);
                if (cb) bp[ij] = transfinite(C, G[2][0].data(), G[2][1].data(), G[2][2].data(), G[2][3].data(), xg[i], xg[j]);
            } else {
                xp[ij] = bilinear(cx, xg[i], xg[j]);
                yp[ij] = bilinear(cy, xg[i], xg[j]);
                if (cb) bp[ij] = bilinear(cb, xg[i], xg[j]);
            }
        }
    element_geometry(e, xp.data(), yp.data());
    if (cb) for (int id = 0; id < n2; ++id) b[(size_t)e * n2 + id] = bp[id];
}

// Structured NX x NY grid over [xL,xR]x[yL,yR] pushed through
//   x -> x + a sin(2 pi kx (x-xL)/Lx) sin(2 pi ky (y-yL)/Ly)   (y likewise),
// every side curved and sampled at m+1 Chebyshev-Lobatto points, i.e. the
// in-memory form of the ISM-V2 file that write_ism2 emits.  rotate != 0
// renumbers element corners by a seeded cyclic shift so that faces of every
// orientation pairing occur (the shipped curved meshes contain such faces).
void Mesh::generate_mapped(double xL, double xR, double yL, double yR, int NX, int NY, double amp,
                           int m, unsigned rotate_seed) {
    const int n = ngl;
    (void)n;
    const double Lx = xR - xL, Ly = yR - yL;
    auto mapxy = [&](double u, double v, double* X, double* Y) {
        const double s = std::sin(2.0 * M_PI * (u - xL) / Lx) * std::sin(2.0 * M_PI * (v - yL) / Ly);
        *X = u + amp * Lx * s;
        *Y = v + amp * Ly * s;
    };
    // nodes (NX+1)*(NY+1), row-major in y.
    const int NN = (NX + 1) * (NY + 1);
    nodes_x.assign(NN, 0.0); nodes_y.assign(NN, 0.0);
    for (int j = 0; j <= NY; ++j)
        for (int i = 0; i <= NX; ++i)
            mapxy(xL + Lx * i / NX, yL + Ly * j / NY, &nodes_x[j * (NX + 1) + i], &nodes_y[j * (NX + 1) + i]);
    // element corner lists, CCW, optionally rotated.
    const int Ke = NX * NY;
    elem_corners.assign((size_t)Ke * 4, 0);
    unsigned st = rotate_seed ? rotate_seed : 1u;
    for (int ey = 0; ey < NY; ++ey)
        for (int ex = 0; ex < NX; ++ex) {
            const int e = ey * NX + ex;
            int c[4] = {ey * (NX + 1) + ex, ey * (NX + 1) + ex + 1, (ey + 1) * (NX + 1) + ex + 1,
                        (ey + 1) * (NX + 1) + ex};
            int r = 0;
            if (rotate_seed) {
                st = st * 1103515245u + 12345u;
                r = (st >> 16) & 3;
            }
            for (int k = 0; k < 4; ++k) elem_corners[(size_t)e * 4 + k] = c[(k + r) & 3];
        }
    curve_order = m;
    elem_curves_stride = 2;
    // curve samples per element side, evaluated from the analytic map along
    // the straight pre-image of the side.
    Curve C;
    C.init(m);
    elem_curves.assign((size_t)Ke * 4 * (m + 1) * 2, 0.0);
    elem_curved.assign((size_t)Ke * 4, 1);
    auto preimage = [&](int node, double* u, double* v) {
        const int i = node % (NX + 1), j = node / (NX + 1);
        *u = xL + Lx * i / NX;
        *v = yL + Ly * j / NY;
    };
    static const int ends[4][2] = {{0, 1}, {1, 2}, {3, 2}, {0, 3}};
    for (int e = 0; e < Ke; ++e)
        for (int s = 0; s < 4; ++s) {
            double ua, va, ub, vb;
            preimage(elem_corners[(size_t)e * 4 + ends[s][0]], &ua, &va);
            preimage(elem_corners[(size_t)e * 4 + ends[s][1]], &ub, &vb);
            for (int k = 0; k <= m; ++k) {
                const double t = 0.5 * (C.xc[k] + 1.0);
                const double u = ua + (ub - ua) * t, v = va + (vb - va) * t;
                double X, Y;
                mapxy(u, v, &X, &Y);
                // snap the end points onto the mapped corner nodes exactly
                if (k == 0) { X = nodes_x[elem_corners[(size_t)e * 4 + ends[s][0]]]; Y = nodes_y[elem_corners[(size_t)e * 4 + ends[s][0]]]; }
                if (k == m) { X = nodes_x[elem_corners[(size_t)e * 4 + ends[s][1]]]; Y = nodes_y[elem_corners[(size_t)e * 4 + ends[s][1]]]; }
                elem_curves[(((size_t)e * 4 + s) * (m + 1) + k) * 2 + 0] = X;
                elem_curves[(((size_t)e * 4 + s) * (m + 1) + k) * 2 + 1] = Y;
            }
        }
    build_from_corner_lists(false);
}

// Builds faces from the element corner lists (each geometric edge once, in
// order of first appearance over elements and sides) and the geometry of all
// elements.  The face records follow the ISM-V2 convention of
// src/Mesh.cpp:782-863: the first element seen is the left one; orientation
// 1 when both elements run their side in the same direction.
void Mesh::build_from_corner_lists(bool has_b) {
    const int Ke = (int)(elem_corners.size() / 4);
    static const int ends[4][2] = {{0, 1}, {1, 2}, {3, 2}, {0, 3}};
    // edge key -> face id via sorted vector of (min,max,face)
    struct Rec { long long key; int e, s; };
    std::vector<Rec> recs;
    recs.reserve((size_t)Ke * 4);
    const long long NNl = (long long)nodes_x.size() + 1;
    for (int e = 0; e < Ke; ++e)
        for (int s = 0; s < 4; ++s) {
            const int a = elem_corners[(size_t)e * 4 + ends[s][0]], b = elem_corners[(size_t)e * 4 + ends[s][1]];
            const long long lo = a < b ? a : b, hi = a < b ? b : a;
            recs.push_back({lo * NNl + hi, e, s});
        }
    std::vector<int> order(recs.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    // stable sort by key keeps (element, side) order inside equal keys
    std::stable_sort(order.begin(), order.end(), [&](int p, int q) { return recs[p].key < recs[q].key; });
    std::vector<int> face_of(recs.size(), -1);
    std::vector<int> first_of_face;
    std::vector<int> second_of_face;
    // assign face ids in order of first appearance
    std::vector<int> group_first(recs.size(), -1);
    for (size_t k = 0; k < order.size();) {
        size_t l = k;
        while (l < order.size() && recs[order[l]].key == recs[order[k]].key) ++l;
        if (l - k > 2) throw std::runtime_error("non-manifold edge in corner lists");
        group_first[order[k]] = order[k];
        if (l - k == 2) group_first[order[k + 1]] = order[k];
        k = l;
    }
    int Fc = 0;
    std::vector<int> fid_of_first(recs.size(), -1);
    for (size_t r = 0; r < recs.size(); ++r) {
        const int g = group_first[r];
        if (g == (int)r) { fid_of_first[r] = Fc++; first_of_face.push_back((int)r); second_of_face.push_back(-1); }
        else second_of_face[fid_of_first[g]] = (int)r;
    }
    std::vector<double> keep_nodes_x = nodes_x, keep_nodes_y = nodes_y, keep_nodes_b = nodes_b;
    alloc(Ke, Fc);
    nodes_x = keep_nodes_x; nodes_y = keep_nodes_y; nodes_b = keep_nodes_b;
    has_bottom = has_b;
    if (has_b) b.assign((size_t)K * ngl * ngl, 0.0);
    for (int f = 0; f < Fc; ++f) {
        const Rec& A = recs[first_of_face[f]];
        int* E = &EdgeInfo[(size_t)f * 7];
        const int a0 = elem_corners[(size_t)A.e * 4 + ends[A.s][0]];
        const int a1 = elem_corners[(size_t)A.e * 4 + ends[A.s][1]];
        E[0] = a0; E[1] = a1; E[2] = A.e; E[4] = A.s;
        ElementToEdge[A.e * 4 + A.s] = f + 1;
        if (second_of_face[f] < 0) { E[3] = -1; E[5] = -1; E[6] = 1; }
        else {
            const Rec& Bq = recs[second_of_face[f]];
            const int b0 = elem_corners[(size_t)Bq.e * 4 + ends[Bq.s][0]];
            E[3] = Bq.e; E[5] = Bq.s;
            E[6] = (b0 == a0) ? 1 : 0;
            ElementToEdge[Bq.e * 4 + Bq.s] = f + 1;
        }
    }
    const int m = curve_order;
    for (int e = 0; e < Ke; ++e) {
        double cx[4], cy[4], cbv[4];
        for (int k = 0; k < 4; ++k) {
            const int nd = elem_corners[(size_t)e * 4 + k];
            cx[k] = nodes_x[nd]; cy[k] = nodes_y[nd];
            cbv[k] = has_b ? nodes_b[nd] : 0.0;
        }
        std::vector<double> gxs[4], gys[4], gbs[4];
        const double* gx[4]; const double* gy[4]; const double* gb[4];
        int cs[4];
        for (int s = 0; s < 4; ++s) {
            cs[s] = elem_curved.empty() ? 0 : elem_curved[(size_t)e * 4 + s];
            gxs[s].assign(m + 1, 0.0); gys[s].assign(m + 1, 0.0); gbs[s].assign(m + 1, 0.0);
            if (cs[s]) {
                const int nc = has_b ? 3 : 2;
                for (int k = 0; k <= m; ++k) {
                    const size_t base = (((size_t)e * 4 + s) * (m + 1) + k) * (size_t)(elem_curves_stride ? elem_curves_stride : 2);
                    gxs[s][k] = elem_curves[base + 0];
                    gys[s][k] = elem_curves[base + 1];
                    if (nc == 3) gbs[s][k] = elem_curves[base + 2];
                }
            }
            gx[s] = gxs[s].data(); gy[s] = gys[s].data(); gb[s] = gbs[s].data();
        }
        element_from_curves(e, cx, cy, has_b ? cbv : nullptr, gx, gy, has_b ? gb : nullptr, cs, m > 0 ? m : 1);
    }
    finish_tables();
}

// ISM-V2 reader (src/Mesh.cpp:698-1503): header, nodes "x y [b]", edges
// "start end elemL elemR sideL sideR" (1-based, negative sideR = reversed),
// per element its corners, curve flags, curve samples and boundary names.
// Unlike the reference the arrays live on the heap, so large meshes need no
// stack-size change.
void Mesh::read_ism2(const std::string& path, bool read_bottom, bool convert_km) {
    std::ifstream in(path);
    if (!in) throw std::invalid_argument("ERROR: Mesh file not found: " + path);
    const double earth_radius = 6.378e3;
    std::string line;
    std::getline(in, line);
    std::getline(in, line);
    int NNd = 0, NE = 0, NK = 0, order = 0;
    {
        std::istringstream ss(line);
        if (!(ss >> NNd >> NE >> NK >> order)) throw std::invalid_argument("ERROR: Header incorrect! " + path);
    }
    auto km = [&](double* X, double* Y) {
        if (convert_km) {
            *X = *X * earth_radius * M_PI / 180.0;
            *Y = earth_radius * std::asinh(std::tan(*Y / 180.0 * M_PI));
        }
    };
    nodes_x.assign(NNd, 0.0); nodes_y.assign(NNd, 0.0); nodes_b.assign(NNd, 0.0);
    for (int i = 0; i < NNd; ++i) {
        std::getline(in, line);
        std::istringstream ss(line);
        if (!(ss >> nodes_x[i] >> nodes_y[i])) throw std::invalid_argument("ERROR: Cant read in Nodes! " + path);
        if (read_bottom && !(ss >> nodes_b[i])) throw std::invalid_argument("ERROR: Cant read in Nodes! " + path);
        km(&nodes_x[i], &nodes_y[i]);
    }
    std::vector<int> edges((size_t)NE * 6);
    for (int is = 0; is < NE; ++is) {
        std::getline(in, line);
        std::istringstream ss(line);
        int* r = &edges[(size_t)is * 6];
        if (!(ss >> r[0] >> r[1] >> r[2] >> r[3] >> r[4] >> r[5]))
            throw std::invalid_argument("ERROR: Cant read in Edge Stuff! " + path);
    }
    curve_order = order;
    const int m = order;
    const int nc = read_bottom ? 3 : 2;
    elem_curves_stride = nc;
    elem_corners.assign((size_t)NK * 4, 0);
    elem_curved.assign((size_t)NK * 4, 0);
    elem_curves.assign((size_t)NK * 4 * (m + 1) * nc, 0.0);
    for (int e = 0; e < NK; ++e) {
        std::getline(in, line);
        {
            std::istringstream ss(line);
            int* c = &elem_corners[(size_t)e * 4];
            if (!(ss >> c[0] >> c[1] >> c[2] >> c[3])) throw std::invalid_argument("ERROR: Cant read in Element Corners! " + path);
            for (int k = 0; k < 4; ++k) c[k] -= 1;
        }
        std::getline(in, line);
        {
            std::istringstream ss(line);
            int* g = &elem_curved[(size_t)e * 4];
            if (!(ss >> g[0] >> g[1] >> g[2] >> g[3])) throw std::invalid_argument("ERROR: Cant read in Gamma information! " + path);
        }
        for (int s = 0; s < 4; ++s) {
            if (!elem_curved[(size_t)e * 4 + s]) continue;
            for (int k = 0; k <= m; ++k) {
                std::getline(in, line);
                std::istringstream ss(line);
                double* v = &elem_curves[(((size_t)e * 4 + s) * (m + 1) + k) * nc];
                if (!(ss >> v[0] >> v[1])) throw std::invalid_argument("ERROR: Cant read in given Gamma Curve! " + path);
                if (nc == 3 && !(ss >> v[2])) throw std::invalid_argument("ERROR: Cant read in given Gamma Curve! " + path);
                km(&v[0], &v[1]);
            }
        }
        std::getline(in, line);  // boundary names
        {
            std::istringstream ss(line);
            std::string nm;
            for (int k = 0; k < 4; ++k)
                if (!(ss >> nm)) throw std::invalid_argument("ERROR: Cant read in given Boundary Names! " + path);
        }
    }
    // Faces as listed in the file.
    alloc(NK, NE);
    has_bottom = read_bottom;
    if (read_bottom) b.assign((size_t)K * ngl * ngl, 0.0);
    for (int is = 0; is < NE; ++is) {
        const int* r = &edges[(size_t)is * 6];
        int* E = &EdgeInfo[(size_t)is * 7];
        E[0] = r[0] - 1; E[1] = r[1] - 1; E[2] = r[2] - 1; E[3] = r[3] - 1; E[4] = r[4] - 1;
        if (E[2] < 0 || E[2] >= NK || E[3] < -1 || E[3] >= NK || E[4] < 0 || E[4] > 3)
            throw std::invalid_argument("ERROR: edge record out of range in " + path);
        ElementToEdge[E[2] * 4 + E[4]] = is + 1;
        if (r[5] < 0) { E[6] = 0; E[5] = -r[5] - 1; }
        else { E[6] = 1; E[5] = r[5] - 1; }
        if (E[3] != -1) {
            if (E[5] < 0 || E[5] > 3) throw std::invalid_argument("ERROR: edge side out of range in " + path);
            ElementToEdge[E[3] * 4 + E[5]] = is + 1;
        }
    }
    for (int e = 0; e < NK; ++e) {
        double cx[4], cy[4], cbv[4];
        for (int k = 0; k < 4; ++k) {
            const int nd = elem_corners[(size_t)e * 4 + k];
            if (nd < 0 || nd >= NNd) throw std::invalid_argument("ERROR: corner id out of range in " + path);
            cx[k] = nodes_x[nd]; cy[k] = nodes_y[nd]; cbv[k] = nodes_b[nd];
        }
        std::vector<double> gxs[4], gys[4], gbs[4];
        const double* gx[4]; const double* gy[4]; const double* gb[4];
        int cs[4];
        for (int s = 0; s < 4; ++s) {
            cs[s] = elem_curved[(size_t)e * 4 + s];
            gxs[s].assign(m + 1, 0.0); gys[s].assign(m + 1, 0.0); gbs[s].assign(m + 1, 0.0);
            if (cs[s])
                for (int k = 0; k <= m; ++k) {
                    const double* v = &elem_curves[(((size_t)e * 4 + s) * (m + 1) + k) * nc];
                    gxs[s][k] = v[0]; gys[s][k] = v[1];
                    if (nc == 3) gbs[s][k] = v[2];
                }
            gx[s] = gxs[s].data(); gy[s] = gys[s].data(); gb[s] = gbs[s].data();
        }
        element_from_curves(e, cx, cy, read_bottom ? cbv : nullptr, gx, gy, read_bottom ? gb : nullptr, cs, m > 0 ? m : 1);
    }
    finish_tables();
}

// ISM-V2 writer for meshes built from corner lists (generate_mapped); the
// output reads back through read_ism2 and through the reference reader.
void Mesh::write_ism2(const std::string& path) const {
    if (elem_corners.empty()) throw std::runtime_error("write_ism2: mesh has no corner lists");
    FILE* fp = std::fopen(path.c_str(), "w");
    if (!fp) throw std::runtime_error("write_ism2: cannot open " + path);
    const int m = curve_order;
    const int stride = elem_curves_stride ? elem_curves_stride : 2;
    std::fprintf(fp, "ISM-V2\n%d %d %d %d\n", (int)nodes_x.size(), F, K, m);
    for (size_t i = 0; i < nodes_x.size(); ++i) std::fprintf(fp, "%.17g %.17g\n", nodes_x[i], nodes_y[i]);
    for (int f = 0; f < F; ++f) {
        const int* E = &EdgeInfo[(size_t)f * 7];
        const int sr = E[3] < 0 ? 0 : (E[6] ? E[5] + 1 : -(E[5] + 1));
        std::fprintf(fp, "%d %d %d %d %d %d\n", E[0] + 1, E[1] + 1, E[2] + 1, E[3] + 1, E[4] + 1, sr);
    }
    for (int e = 0; e < K; ++e) {
        const int* c = &elem_corners[(size_t)e * 4];
        std::fprintf(fp, "%d %d %d %d\n", c[0] + 1, c[1] + 1, c[2] + 1, c[3] + 1);
        const int* g = &elem_curved[(size_t)e * 4];
        std::fprintf(fp, "%d %d %d %d\n", g[0], g[1], g[2], g[3]);
        for (int s = 0; s < 4; ++s) {
            if (!g[s]) continue;
            for (int k = 0; k <= m; ++k) {
                const double* v = &elem_curves[(((size_t)e * 4 + s) * (m + 1) + k) * stride];
                std::fprintf(fp, "%.17g %.17g\n", v[0], v[1]);
            }
        }
        std::fprintf(fp, "--- --- --- ---\n");
    }
    std::fclose(fp);
}

// Packs the arrays handed to the device layer, as src/main.cpp:650-716 does
// for one rank (EdgeData rows from src/MeshPartitioning.cpp:83-130).
void Mesh::pack(PackedMesh* P) const {
    const int n = ngl, n2 = n * n;
    P->K = K; P->F = F; P->ngl = n;
    P->EdgeData.assign((size_t)F * 8, 0);
    P->EdgeReversed.assign(F, 0);
    for (int f = 0; f < F; ++f) {
        const int* E = &EdgeInfo[(size_t)f * 7];
        int* D = &P->EdgeData[(size_t)f * 8];
        D[0] = E[2]; D[1] = E[3]; D[2] = E[4]; D[3] = E[5]; D[4] = E[6];
        D[5] = 0; D[6] = (E[3] == -1) ? -1 : 0; D[7] = f;
        P->EdgeReversed[f] = D[4];
    }
    P->ElemToEdge.assign((size_t)K * 4, 0);
    P->MasterSlave.assign((size_t)K * 4, 0);
    P->Orientation.assign((size_t)K * 4, 0);
    for (int e = 0; e < K; ++e)
        for (int s = 0; s < 4; ++s) {
            const int id = e * 4 + s;
            const int ifa = ElementToEdge[id];
            const int* D = &P->EdgeData[(size_t)(ifa - 1) * 8];
            P->MasterSlave[id] = MasterSlave[id];
            P->Orientation[id] = (D[0] == e) ? 1 : D[4];
            P->ElemToEdge[id] = ifa;
        }
    const size_t nn = (size_t)K * n2;
    P->x = x; P->y = y; P->xXi = xXi; P->xEta = xEta; P->yXi = yXi; P->yEta = yEta;
    P->Jinv.resize(nn);
    for (size_t id = 0; id < nn; ++id) P->Jinv[id] = 1.0 / J[id];
    P->nx = nxFace; P->ny = nyFace; P->scal = scalFace;
    if (has_bottom) P->b = b; else P->b.assign(nn, 0.0);
}

// Split-form bathymetry gradient (src/SW2D.cpp:1048-1105); Jinv = 1/J.
void bottom_derivatives(int K, int n, const double* D0, const double* b, const double* yEta,
                        const double* yXi, const double* xEta, const double* xXi, const double* Jinv,
                        double* Bx, double* By) {
    const int n2 = n * n;
    for (int ie = 0; ie < K; ++ie)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const size_t id = (size_t)ie * n2;
                double B_xi = 0, BYeta_xi = 0, BXxi_eta = 0, B_eta = 0, BYxi_eta = 0, BXeta_xi = 0;
                for (int l = 0; l < n; ++l) {
                    const int il = i * n + l, jl = j * n + l, li = l * n + i;
                    B_xi += D0[il] * b[id + jl];
                    BYeta_xi += D0[il] * b[id + jl] * yEta[id + jl];
                    BXeta_xi += D0[il] * b[id + jl] * xEta[id + jl];
                    B_eta += D0[jl] * b[id + li];
                    BYxi_eta += D0[jl] * b[id + li] * yXi[id + li];
                    BXxi_eta += D0[jl] * b[id + li] * xXi[id + li];
                }
                const size_t xid = id + j * n + i;
                Bx[xid] = 0.5 * Jinv[xid] * (yEta[xid] * B_xi + BYeta_xi - yXi[xid] * B_eta - BYxi_eta);
                By[xid] = 0.5 * Jinv[xid] * (-xEta[xid] * B_xi - BXeta_xi + xXi[xid] * B_eta + BXxi_eta);
            }
}

// Element areas and sqrt of the smallest one (src/basis.cpp:939-966).
double element_sizes(int K, int n, const double* wGL, const double* Jinv, double* EleSize) {
    const int n2 = n * n;
    double mn = 0.0;
    for (int ie = 0; ie < K; ++ie) {
        double s = 0.0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) s += 1.0 / Jinv[(size_t)ie * n2 + j * n + i] * wGL[i] * wGL[j];
        EleSize[ie] = s;
        mn = (ie == 0) ? s : (s < mn ? s : mn);
    }
    return std::sqrt(mn);
}

// Low-storage and SSP Runge-Kutta tables (src/RungeKutta.cpp:18-90); the
// 5-stage 4th-order scheme is Carpenter & Kennedy (1994), solution 3.
int rk_coefficients(int order, int ssp, double* A, double* Bc, double* C) {
    if (order == 3) {
        if (ssp) {
            A[0] = 1.0; A[1] = 3.0 / 4.0; A[2] = 1.0 / 3.0;
            Bc[0] = 0.0; Bc[1] = 1.0 / 4.0; Bc[2] = 2.0 / 3.0;
            C[0] = 1.0; C[1] = 1.0 / 4.0; C[2] = 2.0 / 3.0;
        } else {
            A[0] = 0.0; A[1] = -5.0 / 9.0; A[2] = -153.0 / 128.0;
            Bc[0] = 0.0; Bc[1] = 1.0 / 3.0; Bc[2] = 3.0 / 4.0;
            C[0] = 1.0 / 3.0; C[1] = 15.0 / 16.0; C[2] = 8.0 / 15.0;
        }
        return 3;
    }
    if (order == 4) {
        A[0] = 0.0;
        A[1] = -(567301805773.0 / 1357537059087.0);
        A[2] = -(2404267990393.0 / 2016746695238.0);
        A[3] = -(3550918686646.0 / 2091501179385.0);
        A[4] = -(1275806237668.0 / 842570457699.0);
        Bc[0] = 0.0;
        Bc[1] = (1432997174477.0 / 9575080441755.0);
        Bc[2] = (2526269341429.0 / 6820363962896.0);
        Bc[3] = (2006345519317.0 / 3224310063776.0);
        Bc[4] = (2802321613138.0 / 2924317926251.0);
        C[0] = (1432997174477.0 / 9575080441755.0);
        C[1] = (5161836677717.0 / 13612068292357.0);
        C[2] = (1720146321549.0 / 2090206949498.0);
        C[3] = (3134564353537.0 / 4481467310338.0);
        C[4] = (2277821191437.0 / 14882151754819.0);
        return 5;
    }
    return 0;
}

// Quadrature observables (src/basis.cpp:874-1111).
static inline double entropy_point(double g, double h, double hu, double hv, double b) {
    double u = 0.0, v = 0.0;
    if (h > std::pow(10, -12)) { u = hu / h; v = hv / h; }
    return 0.5 * h * (u * u + v * v) + 0.5 * g * h * h + g * h * b;
}

void diagnostics(int K, int n, const double* wGL, const double* Jinv, const double* q, const double* qref,
                 const double* b, double g, double* L2, double* Linf, double* mass, double* entropy) {
    const int n2 = n * n;
    double l2[3] = {0, 0, 0}, li[3] = {0, 0, 0}, m = 0, S = 0;
    for (int ie = 0; ie < K; ++ie)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const size_t id = (size_t)ie * n2 * 3 + j * n + i, xid = (size_t)ie * n2 + j * n + i;
                const double w = 1.0 / Jinv[xid] * wGL[i] * wGL[j];
                if (qref)
                    for (int eq = 0; eq < 3; ++eq) {
                        const double d = q[id + eq * n2] - qref[id + eq * n2];
                        l2[eq] += std::pow(d, 2) / Jinv[xid] * wGL[i] * wGL[j];
                        li[eq] = std::max(li[eq], std::fabs(d));
                    }
                m += q[id] / Jinv[xid] * wGL[i] * wGL[j];
                S += entropy_point(g, q[id], q[id + n2], q[id + 2 * n2], b ? b[xid] : 0.0) / Jinv[xid] * wGL[i] * wGL[j];
                (void)w;
            }
    for (int eq = 0; eq < 3; ++eq) {
        if (L2) L2[eq] = std::sqrt(l2[eq]);
        if (Linf) Linf[eq] = li[eq];
    }
    if (mass) *mass = m;
    if (entropy) *entropy = S;
}

}  // namespace esdg
