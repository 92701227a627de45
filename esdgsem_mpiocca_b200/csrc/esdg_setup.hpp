// Host-side set-up structures for the ES-DGSEM engine (see esdg_setup.cpp).
#pragma once

#include <string>
#include <vector>

namespace esdg {

struct Basis {
    int N = 0, ngl = 0;
    std::vector<double> xGL, wGL, xG, wG, wbary;
    std::vector<double> D0;       // collocation derivative matrix
    std::vector<double> D;        // flux-differencing matrix 2*D0 + boundary terms
    std::vector<double> Dstrong;  // strong-form matrix D0 + boundary terms
    std::vector<double> Dhat;     // -M^{-1} D0^T M
    std::vector<double> VdmInv;   // nodal -> orthonormal Legendre modes
};

void build_basis(int N, int flux_differencing, Basis* B);
// Boundary-curve sample points -cos(k pi / m), k = 0..m, and their
// barycentric weights (the interpolation of the element sides).
void curve_nodes_weights(int m, double* xc, double* wb);
void lgl_nodes_weights(int N, double* x, double* w);
void gauss_nodes_weights(int N, double* x, double* w);

// Arrays in the layout the device layer consumes (one rank).
struct PackedMesh {
    int K = 0, F = 0, ngl = 0;
    std::vector<int> EdgeData, EdgeReversed, ElemToEdge, MasterSlave, Orientation;
    std::vector<double> x, y, xXi, xEta, yXi, yEta, Jinv, nx, ny, scal, b;
};

struct Mesh {
    explicit Mesh(int N);
    int N, ngl;
    int K = 0, F = 0;
    Basis basis;
    bool has_bottom = false;
    // per-element nodal geometry [K][ngl][ngl] (xi fastest)
    std::vector<double> x, y, xXi, xEta, yXi, yEta, J, b;
    // per element side [K][4][ngl]
    std::vector<double> nxSide, nySide, scalSide;
    // per face [F][ngl] (left element's outward normal)
    std::vector<double> nxFace, nyFace, scalFace;
    // EdgeInfo[F][7] = (startNode, endNode, elemL, elemR, sideL, sideR, sameOrientation)
    std::vector<int> EdgeInfo;
    std::vector<int> ElementToEdge;  // [K][4], 1-based face ids
    std::vector<int> MasterSlave, Orientation;
    // unstructured description (ISM-V2 form)
    std::vector<double> nodes_x, nodes_y, nodes_b;
    std::vector<int> elem_corners, elem_curved;
    std::vector<double> elem_curves;
    int elem_curves_stride = 2;
    int curve_order = 0;

    void alloc(int K, int F);
    void element_geometry(int e, const double* xp, const double* yp);
    void element_from_curves(int e, const double* cx, const double* cy, const double* cb,
                             const double* const* gx, const double* const* gy, const double* const* gb,
                             const int* curved_side, int m);
    void finish_tables();
    void generate_cartesian(double xL, double xR, double yL, double yR, int NX, int NY, bool periodic_wrap_rows,
                            bool periodic_wrap_cols);
    void generate_mapped(double xL, double xR, double yL, double yR, int NX, int NY, double amp, int m,
                         unsigned rotate_seed);
    void build_from_corner_lists(bool has_b);
    void read_ism2(const std::string& path, bool read_bottom, bool convert_km);
    void write_ism2(const std::string& path) const;
    void pack(PackedMesh* P) const;
};

void bottom_derivatives(int K, int n, const double* D0, const double* b, const double* yEta, const double* yXi,
                        const double* xEta, const double* xXi, const double* Jinv, double* Bx, double* By);
double element_sizes(int K, int n, const double* wGL, const double* Jinv, double* EleSize);
int rk_coefficients(int order, int ssp, double* A, double* B, double* C);
void diagnostics(int K, int n, const double* wGL, const double* Jinv, const double* q, const double* qref,
                 const double* b, double g, double* L2, double* Linf, double* mass, double* entropy);

}  // namespace esdg
