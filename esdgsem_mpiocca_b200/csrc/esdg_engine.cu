// Device engine of the B200 ES-DGSEM shallow-water solver and its C ABI.
//
// esdg_deviceclass mirrors the reference's deviceclass (include/deviceclass.h,
// src/deviceclass.cpp): it owns every device buffer, takes the host arrays
// prepared by the set-up code, and runs the time loop.  Differences that are
// design, not behaviour:
//   * dt is computed on the device (wave-speed max by atomicMax on ordered
//     bit patterns), so a step needs no host round trip; the step is captured
//     once into a CUDA graph and replayed; the host polls the done flag every
//     few steps instead of every step.
//   * the edge gather is fused into the face-flux kernel and the volume term,
//     surface lift and RK update into one element kernel per stage.
//   * a non-finite wave speed stops the loop with ESDG_E_NONFINITE instead
//     of running on with NaNs.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/esdg_b200.h"
#include "esdg_kernels.cuh"
#include "esdg_tma.cuh"
#include "esdg_rows.cuh"
#include "esdg_pair.cuh"
#include "esdg_indicator.cuh"
#include "esdg_analysis.cuh"
#include "esdg_geometry.cuh"
#include "esdg_okada.cuh"
#include "esdg_setup.hpp"

namespace esdg {

static thread_local std::string g_create_error;

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
};

// okl/GatherEdgeData/CollectEdgeData_Bottom.okl:16-134 (bathymetry traces, once per run)
__global__ void k_collect_bottom_impl(int F, int ngl, const int* ED, const double* Bv, double* bl, double* br) {
    const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long)F * ngl) return;
    const int f = (int)(gid / ngl), i = (int)(gid % ngl);
    const int* r = ED + (long)f * 8;
    const int n2 = ngl * ngl;
    double vl = 0.0, vr = 0.0;
    if (r[5] == 0) vl = Bv[(long)r[0] * n2 + trace_offset(r[2], i, ngl)];
    if (r[6] == 0) vr = Bv[(long)r[1] * n2 + trace_offset(r[3], i, ngl)];
    if (r[5] == -1) vl = vr;
    if (r[6] == -1) vr = vl;
    bl[gid] = vl;
    br[gid] = vr;
}

// Smallest and largest eigenvalue of V^T V (V n x n, row-major) by cyclic
// Jacobi rotations (Golub & Van Loan, Matrix Computations, sec. 8.5).
static void gram_extremes(const std::vector<double>& V, int n, double* lo, double* hi) {
    std::vector<double> A((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double acc = 0.0;
            for (int k = 0; k < n; ++k) acc += V[(size_t)k * n + i] * V[(size_t)k * n + j];
            A[(size_t)i * n + j] = acc;
        }
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) off += A[(size_t)p * n + q] * A[(size_t)p * n + q];
        if (off < 1e-30) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)p * n + q];
                if (apq == 0.0) continue;
                const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < n; ++k) {  // A <- J^T A J
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = c * akp - sn * akq;
                    A[(size_t)k * n + q] = sn * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = c * apk - sn * aqk;
                    A[(size_t)q * n + k] = sn * apk + c * aqk;
                }
            }
    }
    double mn = A[0], mx = A[0];
    for (int i = 1; i < n; ++i) {
        mn = std::min(mn, A[(size_t)i * n + i]);
        mx = std::max(mx, A[(size_t)i * n + i]);
    }
    *lo = mn;
    *hi = mx;
}

class Engine {
  public:
    // configuration (initDeviceVariables / buildDeviceKernels)
    int N = 0, ngl = 0, K = 0, F = 0, rank = 0, rkSSP = 0, ES = 1, Testcase = 0;
    int PP = 0, AV = 0, DiscBottom = 0, PartialDry = 0, Friction = 0;
    int NumFlux = 0, FluxDiff = 1;
    double eps0 = 0, sigma_max = 0, sigma_min = 0, PosPresTOL = 0, geomFace = 0, g = 9.81, h0 = 0;
    bool inited = false, copied = false, built = false;
    int device = 0;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    std::string err;
    long long launches = 0;
    int kernels_per_step = 0;
    size_t bytes = 0;
    std::vector<Buf> bufs;

    // device buffers
    double *q = nullptr, *gRK = nullptr, *Qt = nullptr, *Qtmp = nullptr;
    double *Jinv = nullptr, *Yxi = nullptr, *Yeta = nullptr, *Xxi = nullptr, *Xeta = nullptr;
    double *Bx = nullptr, *By = nullptr, *B = nullptr, *X = nullptr, *Y = nullptr;
    double *D = nullptr, *Dstrong = nullptr, *Dhat = nullptr, *Vinv = nullptr, *GLw = nullptr, *EleSizes = nullptr;
    double *nx = nullptr, *ny = nullptr, *scal = nullptr, *bL = nullptr, *bR = nullptr, *SP = nullptr;
    double *SGX = nullptr, *SGY = nullptr, *SPV = nullptr, *GX = nullptr, *GY = nullptr, *VP = nullptr;
    int *EdgeData = nullptr;
    int4 *ftab = nullptr, *side = nullptr;
    // analysis outputs per node (initDeviceVariables' CalcArrivalTimes and
    // CalcMaximumElevation; null when off)
    double *arrival = nullptr, *max_elev = nullptr;
    DevState* st = nullptr;
    DevState* st_host = nullptr;  // pinned mirror for polling
    int* elem_inst = nullptr;     // null: one instance
    int I = 1;                    // step-state entries (instances, arena: + one retired slot)

    // Troubled-cell indicator of the artificial-viscosity path: 0 the modal
    // sensor and the viscous terms on every element (the reference's path);
    // 1 the modal sensor with the active set (viscous terms only on flagged
    // elements, same numbers); 2 the learned indicator with the active set
    // (one fused pass where the degree allows, N = 3); 3 the same decisions
    // by three passes (features, network, sensor) at every degree.
    int indicator = 0;
    float* mlpP = nullptr;
    __nv_bfloat16* mlpPb = nullptr;
    float ind_margin = 0.5f;
    double ind_emin = 0.0, ind_emax = 0.0;
    int* act = nullptr;                       // [K + 1]: flags, then the list length
    int* alist = nullptr;                     // [K] flagged elements of the stage
    int4* nbr = nullptr;                      // [K] face neighbours
    __nv_bfloat16* indX = nullptr;            // learned: feature rows [K][kp]
    float *ind_seta = nullptr, *ind_y = nullptr;
    double* ind_energy = nullptr;
    unsigned char* ind_ok = nullptr;
    int mlp_grid = 1;
    int* extent = nullptr;                    // arena: live extent {elements, faces} (null: all)
    unsigned long long* ind_stats = nullptr;  // [4] decision counts
    std::vector<double> Vinv_h;
    std::vector<double> Dfd_h;  // flux-differencing matrix (host copy, row kernel parameter)
    // Testcase 1 (manufactured solution): exact boundary states and source
    // at the stage time t + stage_tfrac dt
    int conv = 0;
    double stage_tfrac = 0.0;
    // partial-dry treatment: per-element dry flag, difference matrices
    int* dry = nullptr;
    double *DcFD = nullptr, *DupFD = nullptr, *DdnFD = nullptr;
    bool pd_copied = false;
    int list_grid = 0;                        // persistent grid of the list kernels
    int face_list_grid = 0;                   // grid of the viscous face kernel over the listed elements' faces
    int ind_grid[3] = {1, 1, 1};              // persistent grids of the indicator (modal, learned, fused)

    // step graph
    cudaGraphExec_t graph = nullptr;
    std::vector<double> gA, gB, gC;
    int gStages = 0;

    ~Engine() { release(); }

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? ESDG_E_NOMEM : ESDG_E_CUDA;
    }

    template <class T>
    int alloc(T** p, size_t n) {
        if (n == 0) n = 1;
        void* v = nullptr;
        cudaError_t e = cudaMalloc(&v, n * sizeof(T));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
        e = cudaMemset(v, 0, n * sizeof(T));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemset");
        bufs.push_back({v, n * sizeof(T)});
        bytes += n * sizeof(T);
        *p = static_cast<T*>(v);
        return 0;
    }

    void release() {
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
        for (auto& e : pev)
            if (e) cudaEventDestroy(e);
        pev.clear();
        for (auto& b : bufs) cudaFree(b.p);
        bufs.clear();
        bytes = 0;
        if (st_host) { cudaFreeHost(st_host); st_host = nullptr; }
        q = gRK = Qt = Qtmp = nullptr;
        mlpP = nullptr; mlpPb = nullptr; act = alist = nullptr; ind_stats = nullptr; nbr = nullptr; extent = nullptr;
        indX = nullptr; ind_seta = ind_y = nullptr; ind_energy = nullptr; ind_ok = nullptr;
        indicator = 0;
        dry = nullptr; DcFD = DupFD = DdnFD = nullptr; pd_copied = false;
        arrival = max_elev = nullptr;
        inited = copied = built = false;
    }

    PhysConst phys() const {
        PhysConst c;
        c.g = g;
        c.half_g = 0.5 * g;
        c.fourth_g = 0.25 * g;
        c.geomFace = geomFace;
        c.PosPresTOL = PosPresTOL;
        c.eps0 = eps0;
        c.sigmaMin = sigma_min;
        c.sigmaMax = sigma_max;
        c.ZeroTOL = std::pow(10.0, -5);
        c.sensor_skip = std::isfinite(sigma_min) ? std::pow(10.0, sigma_min) * (1.0 - 1e-12) : 0.0;
        c.ES = ES;
        return c;
    }

    int init(int N_, int K_, int F_, int rank_, int rkSSP_, int ES_, int Testcase_, double eps0_, double smax,
             double smin, double tol, double geomface, double g_, int PP_, int AV_, int DiscBottom_, double h0_,
             int PartialDry_, int Friction_, int ArrivalTimes_ = 0, int MaxElevation_ = 0) {
        if (inited) release();
        if (N_ < 1 || N_ > 7) return fail(ESDG_E_UNSUPPORTED, "N must be in 1..7");
        if (K_ <= 0 || F_ <= 0) return fail(ESDG_E_ARG, "Nelem and Nfaces must be positive");
        if ((long long)K_ * (N_ + 1) * (N_ + 1) * 3 > (1ll << 31) - 1)
            return fail(ESDG_E_ARG, "Nelem*3*(N+1)^2 must fit a 32-bit int (as in the reference)");
        if (DiscBottom_) return fail(ESDG_E_UNSUPPORTED, "DiscBottom=1 is outside the rebuilt hot path");
        if (Friction_) return fail(ESDG_E_UNSUPPORTED, "FrictionTerms=1 is outside the rebuilt hot path");
        N = N_; ngl = N + 1; K = K_; F = F_; rank = rank_; rkSSP = rkSSP_; ES = ES_; Testcase = Testcase_;
        eps0 = eps0_; sigma_max = smax; sigma_min = smin; PosPresTOL = tol; geomFace = geomface; g = g_;
        PP = PP_; AV = AV_; DiscBottom = DiscBottom_; h0 = h0_; PartialDry = PartialDry_; Friction = Friction_;
        const size_t n2 = (size_t)ngl * ngl, nn = (size_t)K * n2, nd = nn * 3, nf = (size_t)F * ngl;
        int r = 0;
        if ((r = alloc(&q, nd)) || (r = alloc(&gRK, nd)) || (r = alloc(&Qt, nd))) return r;
        if (rkSSP && (r = alloc(&Qtmp, nd))) return r;
        if ((r = alloc(&Jinv, nn)) || (r = alloc(&Yxi, nn)) || (r = alloc(&Yeta, nn)) || (r = alloc(&Xxi, nn)) ||
            (r = alloc(&Xeta, nn)) || (r = alloc(&Bx, nn)) || (r = alloc(&By, nn)) || (r = alloc(&B, nn)) ||
            (r = alloc(&X, nn)) || (r = alloc(&Y, nn)))
            return r;
        if ((r = alloc(&D, n2)) || (r = alloc(&Dstrong, n2)) || (r = alloc(&Dhat, n2)) || (r = alloc(&Vinv, n2)) ||
            (r = alloc(&GLw, (size_t)ngl)) || (r = alloc(&EleSizes, (size_t)K)))
            return r;
        if ((r = alloc(&nx, nf)) || (r = alloc(&ny, nf)) || (r = alloc(&scal, nf)) || (r = alloc(&bL, nf)) ||
            (r = alloc(&bR, nf)) || (r = alloc(&SP, (size_t)K * 12 * ngl)))
            return r;
        if ((r = alloc(&EdgeData, (size_t)F * 8)) || (r = alloc(&ftab, (size_t)F)) || (r = alloc(&side, (size_t)K * 4)))
            return r;
        if (PartialDry) {
            if ((r = alloc(&dry, (size_t)K)) || (r = alloc(&DcFD, n2)) || (r = alloc(&DupFD, n2)) ||
                (r = alloc(&DdnFD, n2)))
                return r;
        }
        if (AV) {
            if ((r = alloc(&SGX, nf * 2)) || (r = alloc(&SGY, nf * 2)) || (r = alloc(&SPV, nf * 2)) ||
                (r = alloc(&GX, nn * 2)) || (r = alloc(&GY, nn * 2)) || (r = alloc(&VP, (size_t)K)))
                return r;
        }
        if (ArrivalTimes_) {
            if ((r = alloc(&arrival, nn))) return r;
            k_fill_f64<<<(unsigned)((nn + 255) / 256), 256>>>(arrival, (long)nn, 1000.0);
            const cudaError_t le = cudaGetLastError();
            if (le != cudaSuccess) return cuda_fail(le, "arrival-time fill");
        }
        if (MaxElevation_ && (r = alloc(&max_elev, nn))) return r;  // from 0, as the reference's calloc
        if ((r = alloc(&st, (size_t)I))) return r;
        cudaError_t e = cudaMallocHost(&st_host, sizeof(DevState));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMallocHost");
        // the zero fills ran on the legacy stream; order them before any
        // copy issued on the engine's non-blocking stream
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
        inited = true;
        return 0;
    }

    template <class T>
    int h2d(T* dst, const T* src, size_t n, const char* name) {
        if (!src) return fail(ESDG_E_ARG, std::string("null host array: ") + name);
        cudaError_t e = cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, name);
        return 0;
    }

    int copy(int PP_, int Nelem, const double* GLw_h, const double* nx_h, const double* ny_h, const double* scal_h,
             const double* yxi_h, const double* yeta_h, const double* xxi_h, const double* xeta_h, const double* b_h,
             const double* Bx_h, const double* By_h, const double* D_h, const double* Ds_h, const double* Dh_h,
             const double* J_h, const double* x_h, const double* y_h, const double* q_h, const double* Es_h,
             const double* gRK_h, const double* Qt_h, const double* Vinv_h_, const int* MS_h, const int* OR_h,
             const int* E2E_h, const int* ED_h, const int* ER_h) {
        if (!inited) return fail(ESDG_E_ARG, "copyDeviceVariables before initDeviceVariables");
        if (Nelem != K) return fail(ESDG_E_ARG, "Nelem differs from initDeviceVariables");
        const size_t n2 = (size_t)ngl * ngl, nn = (size_t)K * n2, nd = nn * 3, nf = (size_t)F * ngl;
        // Validate the connectivity on the host, so that no kernel can index
        // outside its buffers.
        if (!MS_h || !OR_h || !E2E_h || !ED_h || !ER_h) return fail(ESDG_E_ARG, "null connectivity table");
        int r = 0;
        std::vector<int4> ft(F), sd((size_t)K * 4);
        for (int f = 0; f < F; ++f) {
            const int* r = ED_h + (size_t)f * 8;
            const int eL = r[0], eR = r[1], sL = r[2], sR = r[3], same = r[4], cpuL = r[5], cpuR = r[6];
            if (eL < 0 || eL >= K || sL < 0 || sL > 3) return fail(ESDG_E_ARG, "EdgeData: bad left element/side");
            if (cpuL != 0) return fail(ESDG_E_UNSUPPORTED, "EdgeData: left processor must be this rank (0)");
            if (cpuR == -1) {
                ft[f] = make_int4(eL, -1, sL | (same ? 1 : 0) << 4, 0);
            } else {
                if (cpuR != 0) return fail(ESDG_E_UNSUPPORTED, "EdgeData: halo faces need more than one rank");
                if (eR < 0 || eR >= K || sR < 0 || sR > 3) return fail(ESDG_E_ARG, "EdgeData: bad right element/side");
                ft[f] = make_int4(eL, eR, sL | (sR << 2) | ((same ? 1 : 0) << 4), 0);
            }
            if (ER_h[f] != same) return fail(ESDG_E_ARG, "EdgeReversed differs from EdgeData orientation");
        }
        for (int e = 0; e < K; ++e)
            for (int s = 0; s < 4; ++s) {
                const size_t id = (size_t)e * 4 + s;
                const int fc = E2E_h[id] - 1;
                if (fc < 0 || fc >= F) return fail(ESDG_E_ARG, "ElemToEdge: face id out of range");
                const int ms = MS_h[id], orr = OR_h[id];
                if (ms != 1 && ms != -1) return fail(ESDG_E_ARG, "ElemEdgeMasterSlave must be +-1");
                if (orr != 0 && orr != 1) return fail(ESDG_E_ARG, "ElemEdgeOrientation must be 0/1");
                sd[id] = make_int4(fc, ms, orr, 0);
            }
        if ((r = pack_face_flags(ft, sd))) return r;
        if ((r = h2d(nx, nx_h, nf, "normalsX")) || (r = h2d(ny, ny_h, nf, "normalsY")) ||
            (r = h2d(scal, scal_h, nf, "Scal")) || (r = h2d(Yxi, yxi_h, nn, "y_xi")) ||
            (r = h2d(Yeta, yeta_h, nn, "y_eta")) || (r = h2d(Xxi, xxi_h, nn, "x_xi")) ||
            (r = h2d(Xeta, xeta_h, nn, "x_eta")) || (r = h2d(B, b_h, nn, "b")) || (r = h2d(Bx, Bx_h, nn, "Bx")) ||
            (r = h2d(By, By_h, nn, "By")) || (r = h2d(D, D_h, n2, "Dmat")) || (r = h2d(Dstrong, Ds_h, n2, "Dstrong")) ||
            (r = h2d(Dhat, Dh_h, n2, "Dhat")) || (r = h2d(Jinv, J_h, nn, "J")) || (r = h2d(q, q_h, nd, "q")) ||
            (r = h2d(EleSizes, Es_h, (size_t)K, "ElementSizes")) || (r = h2d(Vinv, Vinv_h_, n2, "VdmInv")) ||
            (r = h2d(EdgeData, ED_h, (size_t)F * 8, "EdgeData")) || (r = h2d(ftab, ft.data(), (size_t)F, "faces")) ||
            (r = h2d(side, sd.data(), (size_t)K * 4, "sides")))
            return r;
        if (x_h && (r = h2d(X, x_h, nn, "x_phy"))) return r;
        if (y_h && (r = h2d(Y, y_h, nn, "y_phy"))) return r;
        if (gRK_h && (r = h2d(gRK, gRK_h, nd, "gRK"))) return r;
        if (Qt_h && (r = h2d(Qt, Qt_h, nd, "Qt"))) return r;
        if (PP_ && (r = h2d(GLw, GLw_h, (size_t)ngl, "GLw"))) return r;
        if (!PP_ && GLw_h && (r = h2d(GLw, GLw_h, (size_t)ngl, "GLw"))) return r;
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "copyDeviceVariables");
        Vinv_h.assign(Vinv_h_, Vinv_h_ + n2);
        Dfd_h.assign(D_h, D_h + n2);
        copied = true;
        return 0;
    }

    // Checks that the face records and the element side table describe the
    // same sides (ElemToEdge[e][s] is the face whose record names (e, s)) and
    // packs each face's element-side flags (orientation and MasterSlave of
    // both sides, face_side_flags) into ft[f].w for the face kernel, which
    // writes every face's flux into its elements' side slots.  ft and sd are
    // in one numbering (a single mesh, or one arena instance's ranges).
    int pack_face_flags(std::vector<int4>& ft, const std::vector<int4>& sd, int e_base = 0, int f_base = 0) {
        for (size_t f = 0; f < ft.size(); ++f) {
            int4& t = ft[f];
            const int eL = t.x - e_base, sL = t.z & 3, eR = t.y < 0 ? -1 : t.y - e_base, sR = (t.z >> 2) & 3;
            const int4 l = sd[(size_t)eL * 4 + sL];
            if (l.x - f_base != (int)f) return fail(ESDG_E_ARG, "ElemToEdge of a face's left side names another face");
            int oR = 0, mR = 1;
            if (eR >= 0) {
                const int4 rr = sd[(size_t)eR * 4 + sR];
                if (rr.x - f_base != (int)f)
                    return fail(ESDG_E_ARG, "ElemToEdge of a face's right side names another face");
                oR = rr.z; mR = rr.y;
            }
            t.w = face_side_flags(l.z, l.y, oR, mR);
        }
        return 0;
    }

    int build(int FluxDifferencing, int NumFlux_, int rkSSP_, int AV_, int PP_, int DiscBottom_, int Testcase_) {
        if (!inited) return fail(ESDG_E_ARG, "buildDeviceKernels before initDeviceVariables");
        if (FluxDifferencing != 1)
            return fail(ESDG_E_UNSUPPORTED, "FluxDifferencing=0 (standard DGSEM volume kernel) is not rebuilt");
        if (NumFlux_ != 0 && NumFlux_ != 2 && NumFlux_ != 3)
            return fail(ESDG_E_UNSUPPORTED, "NumFlux must be 0 (ES), 2 (Rusanov-type ES) or 3 (rotated ES)");
        conv = 0;
        switch (Testcase_) {
            case 1:  // manufactured solution: Dirichlet boundary states + source (plain path)
                if (AV_) return fail(ESDG_E_UNSUPPORTED, "Testcase 1 is rebuilt without artificial viscosity");
                conv = 1;
                break;
            case 8: case 88: case 89: case 6: case 32: case 90: case 91:
                return fail(ESDG_E_UNSUPPORTED, "this Testcase needs a boundary kernel other than SolidWalls");
            default: break;
        }
        if (rkSSP_ != rkSSP || AV_ != AV || PP_ != PP || DiscBottom_ != DiscBottom)
            return fail(ESDG_E_ARG, "buildDeviceKernels flags differ from initDeviceVariables");
        NumFlux = NumFlux_;
        FluxDiff = FluxDifferencing;
        int r = 0;
        switch (ngl) {
            case 2: r = setup_tma<2>(); break;
            case 3: r = setup_tma<3>(); break;
            case 4: r = setup_tma<4>(); break;
            case 5: r = setup_tma<5>(); break;
            case 6: r = setup_tma<6>(); break;
            case 7: r = setup_tma<7>(); break;
            case 8: r = setup_tma<8>(); break;
        }
        if (r) return r;
        if (AV) {  // grids of the sensor pass and the list kernels
            switch (ngl) {
                case 2: r = setup_indicator<2>(); break;
                case 3: r = setup_indicator<3>(); break;
                case 4: r = setup_indicator<4>(); break;
                case 5: r = setup_indicator<5>(); break;
                case 6: r = setup_indicator<6>(); break;
                case 7: r = setup_indicator<7>(); break;
                case 8: r = setup_indicator<8>(); break;
            }
            if (r) return r;
        }
        built = true;
        return 0;
    }

    // ---- kernel launchers (dispatch on ngl) ----
    // Blocks of a face-node (or element-warp) kernel over n threads: one pass
    // for a single mesh; for an arena a resident grid that strides over the
    // live extent (the capacity can be far above the live part).
    int face_blocks(long n) {
        const int all = (int)((n + 255) / 256);
        if (!elem_inst) return all;
        if (n_sms <= 0 && cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
            n_sms = 148;
        return std::max(1, std::min(all, n_sms * 4));  // the strided kernels' resident blocks
    }
    int n_sms = 0;

    template <int NGL, bool STRIDE>
    void launch_face_k(const FaceArgs& a, bool av_grad, int blocks) {
        if (av_grad) {
            if (NumFlux == 0) k_face_flux<NGL, 0, true, STRIDE><<<blocks, 256, 0, stream>>>(a);
            else if (NumFlux == 2) k_face_flux<NGL, 2, true, STRIDE><<<blocks, 256, 0, stream>>>(a);
            else k_face_flux<NGL, 3, true, STRIDE><<<blocks, 256, 0, stream>>>(a);
        } else {
            if (NumFlux == 0) k_face_flux<NGL, 0, false, STRIDE><<<blocks, 256, 0, stream>>>(a);
            else if (NumFlux == 2) k_face_flux<NGL, 2, false, STRIDE><<<blocks, 256, 0, stream>>>(a);
            else k_face_flux<NGL, 3, false, STRIDE><<<blocks, 256, 0, stream>>>(a);
        }
    }

    // viscous face flux, one-shot for a single mesh, strided for an arena
    template <int NGL>
    void launch_face_visc(long n, const int* actp, const int* ext) {
        if (elem_inst)
            k_face_visc<NGL, true><<<face_blocks(n), 256, 0, stream>>>(F, ftab, nx, ny, scal, GX, GY, VP, SPV,
                                                                      elem_inst, st, geomFace, actp, ext);
        else
            k_face_visc<NGL, false><<<face_blocks(n), 256, 0, stream>>>(F, ftab, nx, ny, scal, GX, GY, VP, SPV,
                                                                       elem_inst, st, geomFace, actp, ext);
    }

    template <int NGL>
    int launch_face(bool av_grad) {
        FaceArgs a{F, ftab, q, nx, ny, scal, bL, bR, SP, SGX, SGY, elem_inst, st, phys()};
        a.act = (AV && indicator) ? act : nullptr;
        a.extent = extent;
        if (conv) { a.conv = 1; a.tfrac = stage_tfrac; a.X = X; a.Y = Y; }
        const long n = (long)F * NGL;
        const int blocks = face_blocks(n);
        if (elem_inst) launch_face_k<NGL, true>(a, av_grad, blocks);
        else launch_face_k<NGL, false>(a, av_grad, blocks);
        ++launches;
        return 0;
    }

    ElemArgs elem_args(int mode, double A, double Bc, double C, int lam) {
        ElemArgs a;
        a.K = K; a.Jinv = Jinv; a.Yxi = Yxi; a.Yeta = Yeta; a.Xxi = Xxi; a.Xeta = Xeta; a.Bx = Bx; a.By = By;
        a.B = B; a.D = D; a.Dhat = Dhat; a.Dstrong = Dstrong; a.Vinv = Vinv; a.SP = SP; a.SGX = SGX; a.SGY = SGY;
        a.SPV = SPV; a.side = side; a.q = q; a.gRK = gRK; a.Qt = Qt; a.Qtmp = Qtmp; a.GX = GX; a.GY = GY; a.VP = VP;
        a.elem_inst = elem_inst; a.st = st; a.rkA = A; a.rkB = Bc; a.rkC = C; a.mode = mode; a.lam = lam;
        a.c = phys(); a.extent = extent;
        if (PartialDry) {
            a.dry = dry; a.Bn = B; a.Dc = DcFD; a.Dup = DupFD; a.Ddn = DdnFD;
        }
        if (conv) { a.conv = 1; a.tfrac = stage_tfrac; a.X = X; a.Y = Y; }
        a.wait_limit = dbg_wait_limit;
        a.skip_tile = dbg_skip_tile;
        return a;
    }

    // Test hook of the bounded bulk-copy waits (esdg_debug_bulk_wait_test):
    // the wait limit in clock cycles (0: the default) and a tile whose copies
    // are never issued (tile + 1; 0: none).
    long long dbg_wait_limit = 0;
    int dbg_skip_tile = 0;

    int set_bulk_wait_test(long long limit, int skip_tile) {
        if (!built) return fail(ESDG_E_ARG, "bulk-wait test hook before buildDeviceKernels");
        if (limit < 0 || skip_tile < -1) return fail(ESDG_E_ARG, "bulk-wait test hook: limit >= 0, tile >= -1");
        dbg_wait_limit = limit;
        dbg_skip_tile = skip_tile + 1;
        if (graph) return capture_step_graph();
        return 0;
    }

    // Plain-path element kernel: a persistent bulk-copy-pipelined kernel when
    // the element count allows 16-byte bulk granularity, else the one-shot
    // one.  Variants 0..TMA_VARIANTS-1: node-per-thread k_element_tma (CTAs
    // per SM, pipeline depth); then ROW_VARIANTS line-per-thread
    // k_element_rows (elements per tile).  The autotuner times them on the
    // mesh; esdg_set_element_variant can fix one.
    static constexpr int ELEM_VARIANTS = TMA_VARIANTS + ROW_VARIANTS + PAIR_VARIANTS;
    static constexpr int PAIR_FIRST = TMA_VARIANTS + ROW_VARIANTS;  // two-nodes-per-thread variants follow
    int tma_grid[ELEM_VARIANTS] = {};  // persistent grid sizes (0: not usable)
    int tma_ctas[ELEM_VARIANTS] = {};  // resident CTAs per SM
    int tma_variant = 0;
    int forced_variant = -1;
    bool tma_tuned = false;
    float tma_tune_ms[ELEM_VARIANTS] = {};

    template <int NGL, int V>
    int setup_tma_variant() {
        using T = TmaShape<NGL, tma_stages(V)>;
        auto kern = k_element_tma<NGL, tma_min_blocks(V), tma_stages(V)>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_element_tma<NGL, tma_min_blocks(V), tma_stages(V), 0>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_element_tma<NGL, tma_min_blocks(V), tma_stages(V), 2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T::THREADS, T::SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
        const int ntiles = (K + T::NE - 1) / T::NE;
        tma_grid[V] = std::max(1, std::min(ntiles, std::max(per_sm, 1) * sms));
        tma_ctas[V] = per_sm;
        return 0;
    }

    template <int NGL, int R>
    int setup_row_variant() {
        constexpr int NE = row_ne(NGL, R);
        using T = RowShape<NGL, NE, 2>;
        auto kern = k_element_rows<NGL, NE, 2, row_min_blocks(R)>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, T::THREADS, T::SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
        const int ntiles = (K + NE - 1) / NE;
        tma_grid[TMA_VARIANTS + R] = per_sm > 0 ? std::max(1, std::min(ntiles, per_sm * sms)) : 0;
        tma_ctas[TMA_VARIANTS + R] = per_sm;
        return 0;
    }

    // Instance of the node-per-thread and two-nodes-per-thread kernels a
    // launch needs: 0 the plain single mesh, 2 an arena or active set
    // without the partial-dry treatment and manufactured source, 1 all.
    static int elem_gen(const ElemArgs& ea) {
        if (!ea.elem_inst && !ea.extent && !ea.act && !ea.dry && !ea.conv) return 0;
        return (!ea.dry && !ea.conv) ? 2 : 1;
    }

    template <int NGL, int V>
    int setup_pair_variant() {
        using P = PairShape<NGL>;
        auto kern = k_element_pair<NGL, pair_min_blocks(V)>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_element_pair<NGL, pair_min_blocks(V), 0>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::SMEM);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_element_pair<NGL, pair_min_blocks(V), 2>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, P::THREADS, P::SMEM);
        if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
        const int ntiles = (K + P::NE - 1) / P::NE;
        tma_grid[PAIR_FIRST + V] = per_sm > 0 ? std::max(1, std::min(ntiles, per_sm * sms)) : 0;
        tma_ctas[PAIR_FIRST + V] = per_sm;
        return 0;
    }

    template <int NGL, int V>
    void launch_pair_v(const ElemArgs& ea) {
        using P = PairShape<NGL>;
        const int ntiles = (K + P::NE - 1) / P::NE;
        const int gen = elem_gen(ea);
        if (gen == 0)
            k_element_pair<NGL, pair_min_blocks(V), 0><<<tma_grid[PAIR_FIRST + V], P::THREADS, P::SMEM, stream>>>(ea, ntiles);
        else if (gen == 2)
            k_element_pair<NGL, pair_min_blocks(V), 2><<<tma_grid[PAIR_FIRST + V], P::THREADS, P::SMEM, stream>>>(ea, ntiles);
        else
            k_element_pair<NGL, pair_min_blocks(V), 1><<<tma_grid[PAIR_FIRST + V], P::THREADS, P::SMEM, stream>>>(ea, ntiles);
    }

    template <int NGL>
    int setup_tma() {
        using T = TmaShape<NGL>;
        for (auto& g : tma_grid) g = 0;
        for (auto& c : tma_ctas) c = 0;
        tma_tuned = false;
        tma_variant = 0;
        if (((long long)K * T::N2) % 2 != 0) return 0;
        int r = setup_tma_variant<NGL, 0>();
        if (!r) r = setup_tma_variant<NGL, 1>();
        if (!r) r = setup_tma_variant<NGL, 2>();
        if constexpr (row_ngl_ok(NGL)) {
            if (!r) r = setup_row_variant<NGL, 0>();
            if (!r) r = setup_row_variant<NGL, 1>();
        }
        if (!r) r = setup_pair_variant<NGL, 0>();
        if (!r) r = setup_pair_variant<NGL, 1>();
        return r;
    }

    template <int NGL, int V>
    void launch_tma_v(const ElemArgs& ea) {
        using T = TmaShape<NGL, tma_stages(V)>;
        const int ntiles = (K + T::NE - 1) / T::NE;
        // the instance with the branches this step does not need compiled out
        const int gen = elem_gen(ea);
        if (gen == 0)
            k_element_tma<NGL, tma_min_blocks(V), tma_stages(V), 0><<<tma_grid[V], T::THREADS, T::SMEM, stream>>>(ea, ntiles);
        else if (gen == 2)
            k_element_tma<NGL, tma_min_blocks(V), tma_stages(V), 2><<<tma_grid[V], T::THREADS, T::SMEM, stream>>>(ea, ntiles);
        else
            k_element_tma<NGL, tma_min_blocks(V), tma_stages(V), 1><<<tma_grid[V], T::THREADS, T::SMEM, stream>>>(ea, ntiles);
    }

    template <int NGL, int R>
    void launch_rows_v(const ElemArgs& ea) {
        if constexpr (row_ngl_ok(NGL)) {
            constexpr int NE = row_ne(NGL, R);
            using T = RowShape<NGL, NE, 2>;
            DLine<NGL> dm;
            for (int i = 0; i < NGL * NGL; ++i) dm.v[i] = Dfd_h[i];
            const int ntiles = (K + NE - 1) / NE;
            k_element_rows<NGL, NE, 2, row_min_blocks(R)>
                <<<tma_grid[TMA_VARIANTS + R], T::THREADS, T::SMEM, stream>>>(ea, dm, ntiles);
        }
    }

    template <int NGL>
    void launch_tma(const ElemArgs& ea, int v) {
        if (v == 0) launch_tma_v<NGL, 0>(ea);
        else if (v == 1) launch_tma_v<NGL, 1>(ea);
        else if (v == 2) launch_tma_v<NGL, 2>(ea);
        else if (v == TMA_VARIANTS) launch_rows_v<NGL, 0>(ea);
        else if (v == TMA_VARIANTS + 1) launch_rows_v<NGL, 1>(ea);
        else if (v == PAIR_FIRST) launch_pair_v<NGL, 0>(ea);
        else launch_pair_v<NGL, 1>(ea);
    }

    template <int NGL>
    void launch_elem_plain(const ElemArgs& ea) {
        if (tma_grid[tma_variant] > 0) {
            launch_tma<NGL>(ea, tma_variant);
        } else {
            using S = ElemShape<NGL>;
            k_element<NGL><<<(K + S::NE - 1) / S::NE, S::THREADS, 0, stream>>>(ea);
        }
        ++launches;
    }

    // Autotuner: times every variant of the element kernel on this mesh in
    // the step's own update mode, on copies of q and gRK (the state is not
    // touched), and keeps the fastest; runs once, before the step graph is
    // captured.  tune_K: elements to cover (the arena's live extent).
    int tune_K = -1;

    template <int NGL>
    int autotune_tma() {
        if (tma_tuned) return 0;
        tma_tuned = true;
        if (tma_grid[0] <= 0) return 0;
        if (forced_variant >= 0) {
            tma_variant = forced_variant;
            return 0;
        }
        const int Kt = tune_K >= 0 ? tune_K : K;
        if (Kt <= 0) return 0;
        const size_t nd = (size_t)Kt * NGL * NGL * 3;
        // In a step the element kernel follows kernels that evict its inputs
        // from L2, so every timed launch here starts after an L2-sized flush;
        // the variants are interleaved so that none profits from order.
        const size_t flush_bytes = (size_t)256 << 20;
        double *tq = nullptr, *tg = nullptr;
        void* flush = nullptr;
        if (cudaMalloc(&tq, nd * sizeof(double)) != cudaSuccess || cudaMalloc(&tg, nd * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&flush, flush_bytes) != cudaSuccess) {
            cudaFree(tq);
            cudaFree(tg);
            cudaGetLastError();
            tma_tuned = false;  // no room for the copies: keep the default variant
            return 0;
        }
        cudaMemcpyAsync(tq, q, nd * sizeof(double), cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(tg, gRK, nd * sizeof(double), cudaMemcpyDeviceToDevice, stream);
        constexpr int REPS = 5;
        cudaEvent_t ev[ELEM_VARIANTS][REPS][2];
        for (auto& a2 : ev)
            for (auto& b2 : a2)
                for (auto& c2 : b2) cudaEventCreate(&c2);
        const bool have = gStages > 0;
        ElemArgs ea = elem_args(rkSSP ? 1 : 0, have ? gA[0] : 0.0, have ? gB[0] : 1.0, have ? gC[0] : 0.0, 0);
        ea.q = tq;
        ea.gRK = tg;
        for (int v = 0; v < ELEM_VARIANTS; ++v)
            if (tma_grid[v] > 0) launch_tma<NGL>(ea, v);  // first-launch costs
        for (int r = 0; r < REPS; ++r)
            for (int v = 0; v < ELEM_VARIANTS; ++v) {
                if (tma_grid[v] <= 0) continue;
                cudaMemsetAsync(flush, r + v, flush_bytes, stream);
                cudaEventRecord(ev[v][r][0], stream);
                launch_tma<NGL>(ea, v);
                cudaEventRecord(ev[v][r][1], stream);
            }
        cudaError_t e = cudaStreamSynchronize(stream);
        float best = 1e30f;
        for (int v = 0; v < ELEM_VARIANTS && e == cudaSuccess; ++v) {
            if (tma_grid[v] <= 0) continue;
            float sum = 0.0f;
            for (int r = 0; r < REPS && e == cudaSuccess; ++r) {
                float ms = 0.0f;
                e = cudaEventElapsedTime(&ms, ev[v][r][0], ev[v][r][1]);
                sum += ms;
            }
            tma_tune_ms[v] = sum / REPS;
            if (e == cudaSuccess && tma_tune_ms[v] < best) {
                best = tma_tune_ms[v];
                tma_variant = v;
            }
        }
        for (auto& a2 : ev)
            for (auto& b2 : a2)
                for (auto& c2 : b2) cudaEventDestroy(c2);
        cudaFree(tq);
        cudaFree(tg);
        cudaFree(flush);
        if (e != cudaSuccess) return cuda_fail(e, "autotune");
        return 0;
    }

    template <int NGL>
    void launch_stage(int mode, double A, double Bc, double C, bool last, bool shock_stage) {
        using S = ElemShape<NGL>;
        const int eb = (K + S::NE - 1) / S::NE;
        const int lam_in_elem = (last && !PP) ? 1 : 0;
        launch_find_dry<NGL>();
        if (AV && indicator) {
            // active set: indicator (stages > 0; stage 0's runs before the
            // step's dt), plain element kernel (flagged elements only write
            // Qt and are listed), then gradient, viscous face flux and
            // viscous update over the list
            if (shock_stage) {
                if (ind_every_stage || indicator < 2) launch_indicator<NGL>(0);
                else cudaMemsetAsync(act + K, 0, sizeof(int), stream);  // the step's flags, a new list
            }
            launch_face<NGL>(true);
            ElemArgs ea = elem_args(mode, A, Bc, C, lam_in_elem);
            ea.act = act; ea.alist = alist; ea.acount = act + K;
            launch_elem_plain<NGL>(ea);
            k_grad_list<NGL><<<list_grid, S::THREADS, 0, stream>>>(ea);
            // the viscous face fluxes of the listed elements' faces only
            k_face_visc_list<NGL><<<face_list_grid, 256, 0, stream>>>(side, ftab, nx, ny, scal, GX, GY, VP, SPV,
                                                                      elem_inst, st, geomFace, act, alist, act + K);
            k_element_av2<NGL><<<list_grid, S::THREADS, 0, stream>>>(ea);
            launches += 3;
        } else if (!AV) {
            launch_face<NGL>(false);
            launch_elem_plain<NGL>(elem_args(mode, A, Bc, C, lam_in_elem));
        } else {
            // the reference path: the sensor (same arithmetic as okl/ShockCapturing,
            // one entry of the modal transform per thread) then the viscous
            // terms on every element
            if (shock_stage) launch_indicator<NGL>(0);
            launch_face<NGL>(true);
            k_element_av1<NGL><<<eb, S::THREADS, 0, stream>>>(elem_args(2, A, Bc, C, 0));
            const long n = (long)F * NGL;
            launch_face_visc<NGL>(n, nullptr, nullptr);
            k_element_av2<NGL><<<eb, S::THREADS, 0, stream>>>(elem_args(mode, A, Bc, C, lam_in_elem));
            launches += 3;
        }
        if (PP && mode != 2) {
            k_pospres<NGL><<<eb, S::THREADS, 0, stream>>>(K, EleSizes, GLw, Jinv, q, elem_inst, st, last ? 1 : 0,
                                                          phys());
            ++launches;
        }
    }

    template <int NGL>
    void launch_lambda() {
        using S = ElemShape<NGL>;
        k_lambda<NGL><<<(K + S::NE - 1) / S::NE, S::THREADS, 0, stream>>>(K, q, elem_inst, st, phys());
        ++launches;
    }


    template <int NGL>
    void launch_indicator(int stage0) {
        if (indicator) cudaMemsetAsync(act, 0, (size_t)(K + 1) * sizeof(int), stream);
        IndArgs ia;
        ia.K = K; ia.q = q; ia.B = B; ia.Vinv = Vinv; ia.VP = VP; ia.act = indicator ? act : nullptr; ia.nbr = nbr;
        ia.elem_inst = elem_inst; ia.st = st; ia.c = phys(); ia.stage0 = stage0;
        ia.P = mlpP; ia.Pb = mlpPb; ia.L = mlp_layout(NGL); ia.margin = ind_margin;
        ia.emin = ind_emin; ia.emax = ind_emax; ia.stats = ind_stats; ia.extent = extent;
        ia.X = indX; ia.seta = ind_seta; ia.energy = ind_energy; ia.ok = ind_ok; ia.y = ind_y;
        using S = IndShape<NGL>;
        const int ntiles = (K + S::NE - 1) / S::NE;
        if (indicator == 2 && FusedShape<NGL>::OK) {
            if constexpr (FusedShape<NGL>::OK) {
                // features, network and sensor fallback in one pass
                using FS = FusedShape<NGL>;
                const int ftiles = (K + FS::NE - 1) / FS::NE;
                k_indicator_fused<NGL><<<std::min(ftiles, ind_grid[2]), FS::THREADS, 0, stream>>>(ia, ftiles);
                ++launches;
            }
        } else if (indicator >= 2) {
            if constexpr (NGL >= 4 && NGL <= 6) {
                // the network as one batched GEMM over the elements:
                // features, forward pass, then the sensor where unsure
                constexpr int KP = mlp_kp(NGL);
                if constexpr ((32 % (NGL * NGL)) == 0)
                    k_ind_features<NGL><<<std::min(ntiles, ind_grid[0]), S::THREADS, 0, stream>>>(ia, ntiles);
                else
                    k_ind_features_warp<NGL><<<face_blocks((long)K * 32), 256, 0, stream>>>(ia);
                k_mlp_forward<KP><<<mlp_grid, 128, MlpSmem<KP>::fwd_bytes(4), stream>>>(K, indX, mlpP, mlpPb, ind_y,
                                                                                 ia.L, extent);
                k_indicator<NGL, true><<<std::min(ntiles, ind_grid[1]), S::THREADS, 0, stream>>>(ia, ntiles);
                launches += 3;
            }
        } else {
            k_indicator<NGL, false><<<std::min(ntiles, ind_grid[0]), S::THREADS, 0, stream>>>(ia, ntiles);
            ++launches;
        }
    }

    template <int NGL>
    int setup_indicator() {
        using S = ElemShape<NGL>;
        int a2 = 0, gr = 0, sms = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a2, k_element_av2<NGL>, S::THREADS, 0);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&gr, k_grad_list<NGL>, S::THREADS, 0);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return cuda_fail(e, "occupancy (list kernels)");
        list_grid = std::max(1, std::min(std::max(1, std::min(a2, gr)) * sms, (K + S::NE - 1) / S::NE));
        int fv = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fv, k_face_visc_list<NGL>, 256, 0);
        if (e != cudaSuccess) return cuda_fail(e, "occupancy (viscous face list)");
        face_list_grid = std::max(1, std::min(std::max(1, fv) * sms, (int)(((long)K * 4 * NGL + 255) / 256)));
        int o0 = 0, o1 = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o0, k_indicator<NGL, false>, IndShape<NGL>::THREADS, 0);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, k_indicator<NGL, true>, IndShape<NGL>::THREADS, 0);
        if (e != cudaSuccess) return cuda_fail(e, "occupancy (indicator)");
        ind_grid[0] = std::max(1, o0) * sms;
        ind_grid[1] = std::max(1, o1) * sms;
        if constexpr (FusedShape<NGL>::OK) {
            int o2 = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, k_indicator_fused<NGL>, FusedShape<NGL>::THREADS, 0);
            if (e != cudaSuccess) return cuda_fail(e, "occupancy (fused indicator)");
            ind_grid[2] = std::max(1, o2) * sms;
        }
        if constexpr (NGL >= 4 && NGL <= 6) {
            constexpr int KP = mlp_kp(NGL);
            e = cudaFuncSetAttribute(k_mlp_forward<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     MlpSmem<KP>::fwd_bytes(4));
            int om = 0;
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&om, k_mlp_forward<KP>, 128,
                                                                  MlpSmem<KP>::fwd_bytes(4));
            if (e != cudaSuccess) return cuda_fail(e, "occupancy (network)");
            mlp_grid = std::max(1, std::min(std::max(1, om) * sms, (K + 63) / 64));
        }
        return 0;
    }

    // Schedule of the learned indicator (modes 2, 3): every stage, as the
    // reference evaluates its sensor (src/deviceclass.cpp:1043-1046), or
    // once per step, at the step start, the viscosity and the active set
    // then kept for the step's stages.  Modes 0 and 1 (the modal sensor,
    // exact) always run every stage.
    bool ind_every_stage = true;

    int set_indicator_every_stage(int every) {
        if (!inited || !built) return fail(ESDG_E_ARG, "indicator schedule after buildDeviceKernels");
        ind_every_stage = every != 0;
        if (graph) return capture_step_graph();
        return 0;
    }

    // Selects the indicator (0..3; see `indicator`); P (modes 2, 3) is the
    // network's FP32 parameter block of mlp_layout(ngl).total floats.
    int set_indicator(int mode, const float* P_h, int nP, float margin) {
        if (!inited || !built) return fail(ESDG_E_ARG, "set_indicator after buildDeviceKernels");
        if (mode < 0 || mode > 3) return fail(ESDG_E_ARG, "indicator mode must be 0, 1, 2 or 3");
        if (mode > 0 && !AV) return fail(ESDG_E_ARG, "the indicator needs ArtificialViscosity=1");
        if (mode >= 2) {
            if (ngl < 4 || ngl > 6) return fail(ESDG_E_UNSUPPORTED, "the learned indicator supports N = 3..5");
            if (!P_h || nP != mlp_layout(ngl).total)
                return fail(ESDG_E_ARG, "learned indicator: parameter block of " +
                                            std::to_string(mlp_layout(ngl).total) + " floats expected");
            if (!(margin >= 0.0f)) return fail(ESDG_E_ARG, "learned indicator: margin must be >= 0");
        }
        int r = 0;
        if (mode > 0 && !act) {
            if ((r = alloc(&act, (size_t)K + 1)) || (r = alloc(&alist, (size_t)K)) || (r = alloc(&ind_stats, 4)) ||
                (r = alloc(&nbr, (size_t)K)))
                return r;
            // the zero fills ran on the legacy stream
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
            k_build_nbr<<<(K + 255) / 256, 256, 0, stream>>>(0, K, side, ftab, nbr);
        }
        if (mode >= 2) {
            const int n = mlp_layout(ngl).total;
            if (!mlpP) {
                if ((r = alloc(&mlpP, (size_t)n)) || (r = alloc(&mlpPb, (size_t)n)) ||
                    (r = alloc(&indX, (size_t)K * mlp_kp(ngl))) || (r = alloc(&ind_seta, (size_t)K)) ||
                    (r = alloc(&ind_y, (size_t)K)) || (r = alloc(&ind_energy, (size_t)K)) ||
                    (r = alloc(&ind_ok, (size_t)K)))
                    return r;
                cudaError_t e = cudaDeviceSynchronize();
                if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
            }
            cudaError_t e = cudaMemcpyAsync(mlpP, P_h, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, stream);
            if (e != cudaSuccess) return cuda_fail(e, "indicator weights");
            k_mlp_cast<<<(n + 255) / 256, 256, 0, stream>>>(n, mlpP, mlpPb);
            // bounds of the sensor's modal energy n1 = |V m V^T|^2 over the
            // nodal energy |m|^2: squares of the extreme eigenvalues of V^T V
            double lo = 0, hi = 0;
            gram_extremes(Vinv_h, ngl, &lo, &hi);
            ind_emin = lo * lo * (1.0 - 1e-9);
            ind_emax = hi * hi * (1.0 + 1e-9);
            ind_margin = margin;
            e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) return cuda_fail(e, "indicator set-up");
        }
        indicator = mode;
        if (graph) return capture_step_graph();
        return 0;
    }

    int indicator_stats(unsigned long long* out4, int reset) {
        if (!ind_stats) {
            for (int k = 0; k < 4; ++k) out4[k] = 0;
            return 0;
        }
        cudaError_t e = cudaMemcpyAsync(out4, ind_stats, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess && reset) e = cudaMemsetAsync(ind_stats, 0, 4 * sizeof(unsigned long long), stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "indicator stats");
        return 0;
    }

    // Stage time t + fraction * dt (src/deviceclass.cpp:944-952): the LS-RK
    // B coefficients, {0, 1, 1/2} for SSP-RK3.
    double stage_time_fraction(int s) const {
        if (rkSSP) {
            static const double d[3] = {0.0, 1.0, 0.5};
            return s < 3 ? d[s] : 0.0;
        }
        return gB[s];
    }

    // Arrival times / maximum elevation with the step's new time
    // (src/deviceclass.cpp:1130-1141).
    template <int NGL>
    void launch_analysis() {
        if (!arrival && !max_elev) return;
        const long nodes = (long)K * NGL * NGL;
        k_analysis<NGL * NGL><<<(unsigned)((nodes + 255) / 256), 256, 0, stream>>>(nodes, q, B, st, h0, arrival,
                                                                                   max_elev);
        ++launches;
    }

    template <int NGL>
    void launch_step() {
        if (AV) launch_indicator<NGL>(1);
        k_step_begin<<<(I + 127) / 128, 128, 0, stream>>>(I, st, ngl, AV);
        ++launches;
        if (rkSSP) {
            // o_Qtmp.copyFrom(o_q) (src/deviceclass.cpp:933-936)
            cudaMemcpyAsync(Qtmp, q, (size_t)K * ngl * ngl * 3 * sizeof(double), cudaMemcpyDeviceToDevice, stream);
        }
        for (int s = 0; s < gStages; ++s) {
            stage_tfrac = stage_time_fraction(s);
            launch_stage<NGL>(rkSSP ? 1 : 0, gA[s], gB[s], gC[s], s == gStages - 1, s > 0);
        }
        stage_tfrac = 0.0;
        k_step_end<<<(I + 127) / 128, 128, 0, stream>>>(I, st);
        ++launches;
        launch_analysis<NGL>();
    }

#define ESDG_DISPATCH(NGLV, CALL)                 \
    switch (NGLV) {                               \
        case 2: CALL<2>(); break;                 \
        case 3: CALL<3>(); break;                 \
        case 4: CALL<4>(); break;                 \
        case 5: CALL<5>(); break;                 \
        case 6: CALL<6>(); break;                 \
        case 7: CALL<7>(); break;                 \
        case 8: CALL<8>(); break;                 \
        default: break;                           \
    }

    template <int NGL>
    void launch_bottom() {
        k_collect_bottom_impl<<<(F * NGL + 255) / 256, 256, 0, stream>>>(F, NGL, EdgeData, B, bL, bR);
        ++launches;
    }

    int check_ready() {
        if (!inited || !copied || !built) return fail(ESDG_E_ARG, "call initDeviceVariables, copyDeviceVariables and buildDeviceKernels first");
        if (PartialDry && !pd_copied) return fail(ESDG_E_ARG, "PartialDryTreatment=1: call copyPartialDryData first");
        return 0;
    }

    // deviceclass::copyPartialDryData (src/deviceclass.cpp:546-553).
    int copy_partial_dry(const double* Dc, const double* Df, const double* Db) {
        if (!inited) return fail(ESDG_E_ARG, "copyPartialDryData before initDeviceVariables");
        if (!PartialDry) return fail(ESDG_E_ARG, "copyPartialDryData needs PartialDryTreatment=1 at initDeviceVariables");
        if (!Dc || !Df || !Db) return fail(ESDG_E_ARG, "null difference matrix");
        const size_t n2 = (size_t)ngl * ngl;
        int r = 0;
        if ((r = h2d(DcFD, Dc, n2, "DCentralFD")) || (r = h2d(DupFD, Df, n2, "DforwardFD")) ||
            (r = h2d(DdnFD, Db, n2, "DbackwardFD")))
            return r;
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "copyPartialDryData");
        pd_copied = true;
        return 0;
    }

    // FindDryElements of the stage (okl/PartialDryTreatment/FindDryElements.okl).
    template <int NGL>
    void launch_find_dry() {
        if (!PartialDry) return;
        k_find_dry<NGL><<<(K + 255) / 256, 256, 0, stream>>>(K, q, dry, PosPresTOL);
        ++launches;
    }

    // Fixes the element-kernel variant (-1: let the autotuner pick).
    int set_element_variant(int v) {
        if (!built) return fail(ESDG_E_ARG, "set_element_variant before buildDeviceKernels");
        if (v < -1 || v >= ELEM_VARIANTS) return fail(ESDG_E_ARG, "element variant out of range");
        if (v >= 0 && tma_grid[v] <= 0)
            return fail(ESDG_E_UNSUPPORTED, "element variant not available for this degree and element count");
        forced_variant = v;
        tma_tuned = v >= 0;
        if (v >= 0) tma_variant = v;
        if (graph) return capture_step_graph();
        return 0;
    }

    int run_autotune() {
        switch (ngl) {
            case 2: return autotune_tma<2>();
            case 3: return autotune_tma<3>();
            case 4: return autotune_tma<4>();
            case 5: return autotune_tma<5>();
            case 6: return autotune_tma<6>();
            case 7: return autotune_tma<7>();
            case 8: return autotune_tma<8>();
        }
        return 0;
    }

    int capture_step_graph() {
        const long long before = launches;
        cudaGraph_t gr;
        cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
        ESDG_DISPATCH(ngl, launch_step);
        e = cudaStreamEndCapture(stream, &gr);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        // same launch sequence as the executable graph (the usual case: a
        // new time loop with the same settings): update its parameters in
        // place instead of instantiating again
        if (graph) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(graph, gr, &info) == cudaSuccess) {
                cudaGraphDestroy(gr);
                kernels_per_step = (int)(launches - before);
                launches = before;
                return 0;
            }
            cudaGetLastError();
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        e = cudaGraphInstantiate(&graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        kernels_per_step = (int)(launches - before);
        launches = before;
        return 0;
    }

    int poll_state() {
        cudaError_t e = cudaMemcpyAsync(st_host, st, sizeof(DevState), cudaMemcpyDeviceToHost, stream);
        if (e != cudaSuccess) return cuda_fail(e, "state read-back");
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
        return 0;
    }

    // Runs up to nsteps (nsteps <= 0: until done) graph replays.
    int run_steps(long long nsteps) {
        const int chunk = 16;
        long long done_steps = 0;
        for (;;) {
            int r = poll_state();
            if (r) return r;
            if (st_host->done) break;
            long long todo = chunk;
            if (nsteps > 0) {
                if (done_steps >= nsteps) break;
                todo = std::min<long long>(todo, nsteps - done_steps);
            }
            for (long long k = 0; k < todo; ++k) {
                cudaError_t e = cudaGraphLaunch(graph, stream);
                if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
                launches += kernels_per_step;
            }
            done_steps += todo;
        }
        return 0;
    }

    int timeloop(int stages, const double* A, const double* Bc, const double* C, double minEle, double CFL,
                 double DFL, double T, int max_steps, double* t_out, int* steps_out) {
        int r = check_ready();
        if (r) return r;
        if (stages <= 0 || stages > 8 || !A || !Bc || !C) return fail(ESDG_E_ARG, "bad Runge-Kutta tables");
        gA.assign(A, A + stages); gB.assign(Bc, Bc + stages); gC.assign(C, C + stages);
        gStages = stages;
        DevState s0;
        std::memset(&s0, 0, sizeof(s0));
        s0.t = 0.0; s0.T = T; s0.minEle = minEle; s0.CFL = CFL; s0.DFL = DFL;
        s0.max_steps = max_steps;
        s0.pause_on = pause_on; s0.pause_at = pause_at; s0.resume_steps = 0;
        *st_host = s0;
        cudaError_t e = cudaMemcpyAsync(st, st_host, sizeof(DevState), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, "state upload");
        ESDG_DISPATCH(ngl, launch_bottom);
        ESDG_DISPATCH(ngl, launch_lambda);
        if ((r = run_autotune())) return r;
        if ((r = capture_step_graph())) return r;
        if ((r = run_steps(max_steps > 0 ? max_steps : 0))) return r;
        if ((r = poll_state())) return r;
        if (t_out) *t_out = st_host->t;
        if (steps_out) *steps_out = st_host->steps;
        if (st_host->status == ST_NONFINITE)
            return fail(ESDG_E_NONFINITE, "non-finite wave speed: the solution blew up (step " +
                                              std::to_string(st_host->steps) + ")");
        if (st_host->status == ST_TIMEOUT) return fail(ESDG_E_CUDA, "a bulk copy did not complete (bounded wait)");
        return 0;
    }

    // Checkpoint pause of the time loop (esdg_set_pause / esdg_resume).
    int pause_on = 0;
    double pause_at = 0.0;

    int set_pause(double t_pause) {
        pause_on = std::isfinite(t_pause) ? 1 : 0;
        pause_at = pause_on ? t_pause : 0.0;
        return 0;
    }

    // Continues a loop that stopped at a pause: at least one step, then
    // until the next pause, T or the step cap of esdg_dg_timeloop.
    int resume(double* t_out, int* steps_out) {
        int r = check_ready();
        if (r) return r;
        if (!graph) return fail(ESDG_E_ARG, "esdg_resume needs a previous esdg_dg_timeloop call");
        if ((r = poll_state())) return r;
        const bool finished = !(st_host->t < st_host->T) ||
                              (st_host->max_steps > 0 && st_host->steps >= st_host->max_steps) ||
                              st_host->status != ST_OK;
        if (!finished) {
            st_host->done = 0;
            st_host->pause_on = pause_on;
            st_host->pause_at = pause_at;
            st_host->resume_steps = st_host->steps;
            cudaError_t e = cudaMemcpyAsync(st, st_host, sizeof(DevState), cudaMemcpyHostToDevice, stream);
            if (e != cudaSuccess) return cuda_fail(e, "state upload");
            if ((r = run_steps(0))) return r;
            if ((r = poll_state())) return r;
        }
        if (t_out) *t_out = st_host->t;
        if (steps_out) *steps_out = st_host->steps;
        if (st_host->status == ST_NONFINITE)
            return fail(ESDG_E_NONFINITE, "non-finite wave speed: the solution blew up (step " +
                                              std::to_string(st_host->steps) + ")");
        if (st_host->status == ST_TIMEOUT) return fail(ESDG_E_CUDA, "a bulk copy did not complete (bounded wait)");
        return 0;
    }

    int advance(int nsteps, double T, double* t_out, int* steps_out) {
        int r = check_ready();
        if (r) return r;
        if (!graph) return fail(ESDG_E_ARG, "esdg_advance needs a previous esdg_dg_timeloop call");
        if ((r = poll_state())) return r;
        st_host->T = T;
        st_host->done = 0;
        st_host->max_steps = 0;
        cudaError_t e = cudaMemcpyAsync(st, st_host, sizeof(DevState), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, "state upload");
        // Enough replays for nsteps; the step cap makes extra replays no-ops.
        const int target = st_host->steps + nsteps;
        st_host->max_steps = target;
        e = cudaMemcpyAsync(st, st_host, sizeof(DevState), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, "state upload");
        for (int k = 0; k < nsteps; ++k) {
            e = cudaGraphLaunch(graph, stream);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
            launches += kernels_per_step;
        }
        if ((r = poll_state())) return r;
        if (t_out) *t_out = st_host->t;
        if (steps_out) *steps_out = st_host->steps;
        if (st_host->status == ST_NONFINITE) return fail(ESDG_E_NONFINITE, "non-finite wave speed");
        if (st_host->status == ST_TIMEOUT) return fail(ESDG_E_CUDA, "a bulk copy did not complete (bounded wait)");
        return 0;
    }

    // Real steps launched one kernel at a time with CUDA events recorded on
    // the launching stream around the face and element launches; returns the
    // average duration of each (for roofline reporting).
    int prof_stage_index = -1;
    // per profiled stage: before the face kernel, between the face and the
    // element kernels, after the element kernel(s); read after the last
    // step, so the kernels stay queued back to back as in the step graph
    std::vector<cudaEvent_t> pev;

    template <int NGL>
    void launch_step_profiled(cudaEvent_t* pe) {
        if (AV) launch_indicator<NGL>(1);
        k_step_begin<<<(I + 127) / 128, 128, 0, stream>>>(I, st, ngl, AV);
        ++launches;
        if (rkSSP)
            cudaMemcpyAsync(Qtmp, q, (size_t)K * ngl * ngl * 3 * sizeof(double), cudaMemcpyDeviceToDevice, stream);
        using S = ElemShape<NGL>;
        const int eb = (K + S::NE - 1) / S::NE;
        for (int s = 0; s < gStages; ++s) {
            const bool last = s == gStages - 1;
            const int mode = rkSSP ? 1 : 0;
            const int lam_in_elem = (last && !PP) ? 1 : 0;
            stage_tfrac = stage_time_fraction(s);
            launch_find_dry<NGL>();
            cudaEvent_t* ev = pe + 3 * s;
            cudaEventRecord(ev[0], stream);
            launch_face<NGL>(AV != 0);
            cudaEventRecord(ev[1], stream);
            if (!AV) {
                launch_elem_plain<NGL>(elem_args(mode, gA[s], gB[s], gC[s], lam_in_elem));
            } else {
                if (s > 0) launch_indicator<NGL>(0);
                k_element_av1<NGL><<<eb, S::THREADS, 0, stream>>>(elem_args(2, gA[s], gB[s], gC[s], 0));
                const long n = (long)F * NGL;
                launch_face_visc<NGL>(n, nullptr, nullptr);
                k_element_av2<NGL><<<eb, S::THREADS, 0, stream>>>(elem_args(mode, gA[s], gB[s], gC[s], lam_in_elem));
                launches += 3;
            }
            cudaEventRecord(ev[2], stream);
            if (PP) {
                k_pospres<NGL><<<eb, S::THREADS, 0, stream>>>(K, EleSizes, GLw, Jinv, q, elem_inst, st, last ? 1 : 0,
                                                              phys());
                ++launches;
            }
        }
        stage_tfrac = 0.0;
        k_step_end<<<(I + 127) / 128, 128, 0, stream>>>(I, st);
        ++launches;
        launch_analysis<NGL>();
    }

    int profile_steps(int nsteps, double* face_ms, double* elem_ms) {
        int r = check_ready();
        if (r) return r;
        if (gStages <= 0) return fail(ESDG_E_ARG, "profile_steps needs a previous esdg_dg_timeloop call");
        if (AV && indicator) return fail(ESDG_E_UNSUPPORTED, "profile_steps times the reference path (indicator 0)");
        const size_t nev = (size_t)nsteps * gStages * 3;
        while (pev.size() < nev) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreate(&e) != cudaSuccess) return fail(ESDG_E_CUDA, "cudaEventCreate");
            pev.push_back(e);
        }
        if ((r = poll_state())) return r;
        st_host->done = 0;
        st_host->max_steps = 0;
        st_host->T = 1e300;
        cudaError_t e = cudaMemcpyAsync(st, st_host, sizeof(DevState), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, "state upload");
        for (int k = 0; k < nsteps; ++k) {
            cudaEvent_t* pe = pev.data() + (size_t)k * gStages * 3;
            switch (ngl) {
                case 2: launch_step_profiled<2>(pe); break;
                case 3: launch_step_profiled<3>(pe); break;
                case 4: launch_step_profiled<4>(pe); break;
                case 5: launch_step_profiled<5>(pe); break;
                case 6: launch_step_profiled<6>(pe); break;
                case 7: launch_step_profiled<7>(pe); break;
                case 8: launch_step_profiled<8>(pe); break;
            }
        }
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "profile_steps");
        double f = 0, el = 0;
        for (size_t k = 0; k < nev; k += 3) {
            float a = 0, b = 0;
            cudaEventElapsedTime(&a, pev[k], pev[k + 1]);
            cudaEventElapsedTime(&b, pev[k + 1], pev[k + 2]);
            f += a;
            el += b;
        }
        const double nl = (double)nsteps * gStages;
        *face_ms = f / nl;
        *elem_ms = el / nl;
        return 0;
    }

    template <int NGL>
    void launch_rhs() {
        stage_tfrac = 0.0;  // one RHS at the state's own time
        if (AV) {
            // the sensor of this state (whatever the learned schedule), then
            // the stage
            launch_indicator<NGL>(0);
            launch_stage<NGL>(2, 0.0, 0.0, 0.0, false, false);
        } else {
            launch_stage<NGL>(2, 0.0, 0.0, 0.0, false, false);
        }
    }

    int rhs(double* Qt_h, double* visc_h) {
        int r = check_ready();
        if (r) return r;
        DevState s0;
        std::memset(&s0, 0, sizeof(s0));
        s0.T = 1.0;
        *st_host = s0;
        cudaError_t e = cudaMemcpyAsync(st, st_host, sizeof(DevState), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cuda_fail(e, "state upload");
        ESDG_DISPATCH(ngl, launch_bottom);
        ESDG_DISPATCH(ngl, launch_rhs);
        const size_t nd = (size_t)K * ngl * ngl * 3;
        e = cudaMemcpyAsync(Qt_h, Qt, nd * sizeof(double), cudaMemcpyDeviceToHost, stream);
        if (e != cudaSuccess) return cuda_fail(e, "Qt read-back");
        if (AV && visc_h) {
            e = cudaMemcpyAsync(visc_h, VP, (size_t)K * sizeof(double), cudaMemcpyDeviceToHost, stream);
            if (e != cudaSuccess) return cuda_fail(e, "visc read-back");
        }
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "compute_rhs");
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "compute_rhs launch");
        return 0;
    }
};

}  // namespace esdg

// ===========================================================================
// C ABI
// ===========================================================================
struct esdg_deviceclass {
    esdg::Engine eng;
};

struct esdg_mesh {
    esdg::Mesh m;
    explicit esdg_mesh(int N) : m(N) {}
};

#define ESDG_GUARD(d)                                          \
    if (!(d)) return ESDG_E_ARG;                               \
    cudaError_t _dev_e = cudaSetDevice((d)->eng.device);       \
    if (_dev_e != cudaSuccess) return (d)->eng.cuda_fail(_dev_e, "cudaSetDevice");

extern "C" {

int esdg_deviceclass_create(int rank, int device_id, esdg_deviceclass** out) {
    if (!out) return ESDG_E_ARG;
    *out = nullptr;
    int dev = device_id;
    cudaError_t e;
    if (dev < 0) {
        e = cudaGetDevice(&dev);
        if (e != cudaSuccess) { esdg::g_create_error = cudaGetErrorString(e); return ESDG_E_CUDA; }
    }
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) { esdg::g_create_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e); return ESDG_E_CUDA; }
    esdg_deviceclass* d = new (std::nothrow) esdg_deviceclass();
    if (!d) return ESDG_E_NOMEM;
    d->eng.device = dev;
    d->eng.rank = rank;
    e = cudaStreamCreateWithFlags(&d->eng.own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        esdg::g_create_error = std::string("cudaStreamCreate: ") + cudaGetErrorString(e);
        delete d;
        return ESDG_E_CUDA;
    }
    d->eng.stream = d->eng.own_stream;
    *out = d;
    return ESDG_OK;
}

int esdg_init_device_variables(esdg_deviceclass* d, int N, int Nelem, int Nfaces, int rank, int rkSSP, int NEpad,
                               int NEsurfpad, int Nedgepad, int NAvgPad, int ES, int Testcase, double epsilon_0,
                               double sigma_max, double sigma_min, double PosPresTOL, double geomface,
                               double g_const, int PositivityPreserving, int ArtificialViscosity, int DiscBottom,
                               double h_0, int PartialDry, int FrictionTerms, int CalcArrivalTimes,
                               int CreateTimeSeries, int CalcMaximumElevation) {
    ESDG_GUARD(d);
    (void)NEpad; (void)NEsurfpad; (void)Nedgepad; (void)NAvgPad;  // launch shapes are chosen per ngl
    (void)CreateTimeSeries;  // gauge series: written by the C++ facade at the plot checkpoints
    return d->eng.init(N, Nelem, Nfaces, rank, rkSSP, ES, Testcase, epsilon_0, sigma_max, sigma_min, PosPresTOL,
                       geomface, g_const, PositivityPreserving, ArtificialViscosity, DiscBottom, h_0, PartialDry,
                       FrictionTerms, CalcArrivalTimes, CalcMaximumElevation);
}

int esdg_copy_device_variables(esdg_deviceclass* d, int PositivityPreserving, int Nelem, const double* GLw,
                               const double* normalsX, const double* normalsY, const double* Scal,
                               const double* y_xi, const double* y_eta, const double* x_xi, const double* x_eta,
                               const double* b, const double* Bx, const double* By, const double* Dmat,
                               const double* Dstrong, const double* Dhat, const double* J, const double* x_phy,
                               const double* y_phy, const double* q, const double* ElementSizes, const double* gRK,
                               const double* Qt, const double* VdmInv, const int* ElemEdgeMasterSlave,
                               const int* ElemEdgeOrientation, const int* ElemToEdge, const int* EdgeData,
                               const int* EdgeReversed) {
    ESDG_GUARD(d);
    return d->eng.copy(PositivityPreserving, Nelem, GLw, normalsX, normalsY, Scal, y_xi, y_eta, x_xi, x_eta, b, Bx,
                       By, Dmat, Dstrong, Dhat, J, x_phy, y_phy, q, ElementSizes, gRK, Qt, VdmInv,
                       ElemEdgeMasterSlave, ElemEdgeOrientation, ElemToEdge, EdgeData, EdgeReversed);
}

int esdg_copy_partial_dry_data(esdg_deviceclass* d, const double* DCentralFD, const double* DforwardFD,
                               const double* DbackwardFD) {
    ESDG_GUARD(d);
    return d->eng.copy_partial_dry(DCentralFD, DforwardFD, DbackwardFD);
}

int esdg_build_device_kernels(esdg_deviceclass* d, int KernelVersion, int KernelVersionSTD, int Testcase,
                              int FluxDifferencing, int NumFlux, int rkSSP, int ArtificialViscosity,
                              int PositivityPreserving, int DiscBottom) {
    ESDG_GUARD(d);
    (void)KernelVersion; (void)KernelVersionSTD;
    return d->eng.build(FluxDifferencing, NumFlux, rkSSP, ArtificialViscosity, PositivityPreserving, DiscBottom,
                        Testcase);
}

int esdg_dg_timeloop(esdg_deviceclass* d, int Nelem, int Nfaces, int rkStages, const double* rkA, const double* rkB,
                     const double* rkC, double globalMinEleSize, double CFL, double DFL, double T, int Testcase,
                     int ArtificialViscosity, int rkSSP, int NumPlots, int NumTimeChecks, double g_const,
                     int PlotVar, int EntropyPlot, int PositivityPreserving, int DiscBottom, int max_steps,
                     double* t_out, int* steps_out) {
    ESDG_GUARD(d);
    // plot outputs are the C++ facade's (checkpoints through esdg_set_pause / esdg_resume)
    (void)NumPlots; (void)NumTimeChecks; (void)PlotVar; (void)EntropyPlot; (void)Testcase;
    esdg::Engine& E = d->eng;
    if (Nelem != E.K || Nfaces != E.F) return E.fail(ESDG_E_ARG, "Nelem/Nfaces differ from initDeviceVariables");
    if (ArtificialViscosity != E.AV || rkSSP != E.rkSSP || PositivityPreserving != E.PP || DiscBottom != E.DiscBottom)
        return E.fail(ESDG_E_ARG, "time-loop flags differ from initDeviceVariables");
    if (g_const != E.g) return E.fail(ESDG_E_ARG, "g_const differs from initDeviceVariables");
    return E.timeloop(rkStages, rkA, rkB, rkC, globalMinEleSize, CFL, DFL, T, max_steps, t_out, steps_out);
}

int esdg_copy_q_to_host(esdg_deviceclass* d, double* q) {
    ESDG_GUARD(d);
    esdg::Engine& E = d->eng;
    if (!E.inited || !q) return E.fail(ESDG_E_ARG, "copy_q_to_host: not initialised or null");
    cudaError_t e = cudaMemcpyAsync(q, E.q, (size_t)E.K * E.ngl * E.ngl * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                    E.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
    if (e != cudaSuccess) return E.cuda_fail(e, "copy_q_to_host");
    return ESDG_OK;
}

int esdg_copy_q_from_host(esdg_deviceclass* d, const double* q) {
    ESDG_GUARD(d);
    esdg::Engine& E = d->eng;
    if (!E.inited || !q) return E.fail(ESDG_E_ARG, "copy_q_from_host: not initialised or null");
    cudaError_t e = cudaMemcpyAsync(E.q, q, (size_t)E.K * E.ngl * E.ngl * 3 * sizeof(double), cudaMemcpyHostToDevice,
                                    E.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
    if (e != cudaSuccess) return E.cuda_fail(e, "copy_q_from_host");
    return ESDG_OK;
}

int esdg_copy_visc_to_host(esdg_deviceclass* d, double* visc) {
    ESDG_GUARD(d);
    esdg::Engine& E = d->eng;
    if (!E.inited || !E.AV || !visc) return E.fail(ESDG_E_ARG, "copy_visc_to_host: AV not enabled or null");
    cudaError_t e = cudaMemcpyAsync(visc, E.VP, (size_t)E.K * sizeof(double), cudaMemcpyDeviceToHost, E.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
    if (e != cudaSuccess) return E.cuda_fail(e, "copy_visc_to_host");
    return ESDG_OK;
}

static int copy_analysis(esdg_deviceclass* d, const double* src, double* out, const char* what) {
    esdg::Engine& E = d->eng;
    if (!E.inited || !src || !out)
        return E.fail(ESDG_E_ARG, std::string(what) + ": not enabled at initDeviceVariables, or null");
    cudaError_t e = cudaMemcpyAsync(out, src, (size_t)E.K * E.ngl * E.ngl * sizeof(double), cudaMemcpyDeviceToHost,
                                    E.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
    if (e != cudaSuccess) return E.cuda_fail(e, what);
    return ESDG_OK;
}

int esdg_copy_arrival_times(esdg_deviceclass* d, double* arrival_times) {
    ESDG_GUARD(d);
    return copy_analysis(d, d->eng.arrival, arrival_times, "copy_arrival_times");
}

int esdg_copy_maximum_elevation(esdg_deviceclass* d, double* maximum_elevation) {
    ESDG_GUARD(d);
    return copy_analysis(d, d->eng.max_elev, maximum_elevation, "copy_maximum_elevation");
}

long long esdg_bytes_allocated(const esdg_deviceclass* d) { return d ? (long long)d->eng.bytes : -1; }

long long esdg_kernel_launches(const esdg_deviceclass* d) { return d ? d->eng.launches : -1; }

int esdg_free_occa_vars(esdg_deviceclass* d, int rkSSP, int PositivityPreserving, int ArtificialViscosity) {
    ESDG_GUARD(d);
    (void)rkSSP; (void)PositivityPreserving; (void)ArtificialViscosity;
    d->eng.release();
    return ESDG_OK;
}

int esdg_deviceclass_destroy(esdg_deviceclass* d) {
    if (!d) return ESDG_E_ARG;
    cudaSetDevice(d->eng.device);
    d->eng.release();
    if (d->eng.own_stream) cudaStreamDestroy(d->eng.own_stream);
    delete d;
    return ESDG_OK;
}

const char* esdg_last_error(const esdg_deviceclass* d) {
    return d ? d->eng.err.c_str() : esdg::g_create_error.c_str();
}

int esdg_compute_rhs(esdg_deviceclass* d, double* Qt_host, double* visc_host) {
    ESDG_GUARD(d);
    if (!Qt_host) return d->eng.fail(ESDG_E_ARG, "null Qt");
    return d->eng.rhs(Qt_host, visc_host);
}

int esdg_set_indicator(esdg_deviceclass* d, int mode, const float* params, int nparams, float margin) {
    ESDG_GUARD(d);
    return d->eng.set_indicator(mode, params, nparams, margin);
}

int esdg_set_indicator_every_stage(esdg_deviceclass* d, int every_stage) {
    ESDG_GUARD(d);
    return d->eng.set_indicator_every_stage(every_stage);
}

int esdg_indicator_stats(esdg_deviceclass* d, unsigned long long* counts4, int reset) {
    ESDG_GUARD(d);
    if (!counts4) return d->eng.fail(ESDG_E_ARG, "null counts");
    return d->eng.indicator_stats(counts4, reset);
}

int esdg_tuned_config(const esdg_deviceclass* d, int* ctas_per_sm, int* stages, float* ms_variants3) {
    if (!d) return ESDG_E_ARG;
    const esdg::Engine& E = d->eng;
    const int v = E.tma_variant;
    const bool node_kernel = v < esdg::TMA_VARIANTS;
    if (ctas_per_sm) *ctas_per_sm = E.tma_grid[v] > 0 ? (node_kernel ? esdg::tma_min_blocks(v) : E.tma_ctas[v]) : 0;
    if (ms_variants3)
        for (int k = 0; k < esdg::TMA_VARIANTS; ++k) ms_variants3[k] = E.tma_tune_ms[k];
    if (stages) *stages = E.tma_grid[v] > 0 ? (node_kernel ? esdg::tma_stages(v) : 2) : 0;
    return E.tma_tuned ? ESDG_OK : ESDG_E_ARG;
}

static int element_variants(const esdg::Engine& E, int* chosen, int* count, float* ms, int* ctas, int cap) {
    constexpr int NV = esdg::Engine::ELEM_VARIANTS;
    if (count) *count = NV;
    if (chosen) *chosen = E.tma_grid[E.tma_variant] > 0 ? E.tma_variant : -1;
    for (int k = 0; k < NV && k < cap; ++k) {
        if (ms) ms[k] = E.tma_tune_ms[k];
        if (ctas) ctas[k] = E.tma_grid[k] > 0 ? E.tma_ctas[k] : 0;
    }
    return E.tma_tuned ? ESDG_OK : ESDG_E_ARG;
}

int esdg_element_variants(const esdg_deviceclass* d, int* chosen, int* count, float* ms, int* ctas_per_sm,
                          int cap) {
    if (!d) return ESDG_E_ARG;
    return element_variants(d->eng, chosen, count, ms, ctas_per_sm, cap);
}

int esdg_set_element_variant(esdg_deviceclass* d, int variant) {
    ESDG_GUARD(d);
    return d->eng.set_element_variant(variant);
}

int esdg_state_pointers(esdg_deviceclass* d, const double** q, const double** b, const double** VdmInv) {
    ESDG_GUARD(d);
    if (!d->eng.built) return d->eng.fail(ESDG_E_ARG, "state_pointers before buildDeviceKernels");
    if (q) *q = d->eng.q;
    if (b) *b = d->eng.B;
    if (VdmInv) *VdmInv = d->eng.Vinv;
    return ESDG_OK;
}

int esdg_set_stream(esdg_deviceclass* d, void* cuda_stream) {
    ESDG_GUARD(d);
    esdg::Engine& E = d->eng;
    E.stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : E.own_stream;
    if (E.graph) { cudaGraphExecDestroy(E.graph); E.graph = nullptr; }
    return ESDG_OK;
}

int esdg_profile_steps(esdg_deviceclass* d, int nsteps, double* face_ms, double* elem_ms) {
    ESDG_GUARD(d);
    if (nsteps <= 0 || nsteps > 1000 || !face_ms || !elem_ms)
        return d->eng.fail(ESDG_E_ARG, "bad profile_steps arguments");
    return d->eng.profile_steps(nsteps, face_ms, elem_ms);
}

int esdg_set_pause(esdg_deviceclass* d, double t_pause) {
    if (!d) return ESDG_E_ARG;
    return d->eng.set_pause(t_pause);
}

int esdg_resume(esdg_deviceclass* d, double* t_out, int* steps_out) {
    if (!d) return ESDG_E_ARG;
    return d->eng.resume(t_out, steps_out);
}

int esdg_debug_bulk_wait_test(esdg_deviceclass* d, long long wait_limit_cycles, int skip_tile) {
    if (!d) return ESDG_E_ARG;
    return d->eng.set_bulk_wait_test(wait_limit_cycles, skip_tile);
}

int esdg_advance(esdg_deviceclass* d, int nsteps, double T, double* t_out, int* steps_out) {
    ESDG_GUARD(d);
    if (nsteps < 0) return d->eng.fail(ESDG_E_ARG, "nsteps < 0");
    if (!d->eng.graph) {
        if (d->eng.gStages <= 0) return d->eng.fail(ESDG_E_ARG, "esdg_advance needs a previous esdg_dg_timeloop call");
        int r = d->eng.capture_step_graph();
        if (r) return r;
    }
    return d->eng.advance(nsteps, T, t_out, steps_out);
}

// ---------------------------------------------------------------------------
// Set-up
// ---------------------------------------------------------------------------
int esdg_basis_fd(int N, double* Dc, double* Df, double* Db) {
    // src/basis.cpp:190-229: two-point differences on the LGL nodes; row i of
    // each matrix holds the weights of node i's difference (all other
    // entries zero).  Central: one-sided at the two ends.
    if (N < 1 || N > 15 || !Dc || !Df || !Db) return ESDG_E_ARG;
    std::vector<double> x(N + 1), w(N + 1);
    esdg::lgl_nodes_weights(N, x.data(), w.data());
    const int n = N + 1, n2 = n * n;
    for (int k = 0; k < n2; ++k) Dc[k] = Df[k] = Db[k] = 0.0;
    const double first = 1.0 / (x[1] - x[0]), last = 1.0 / (x[N] - x[N - 1]);
    Dc[0] = -first; Dc[1] = first;
    Dc[n2 - 2] = -last; Dc[n2 - 1] = last;
    for (int i = 1; i + 1 < n; ++i) {
        const double c = 1.0 / (x[i + 1] - x[i - 1]);
        Dc[i * n + i - 1] = -c;
        Dc[i * n + i + 1] = c;
    }
    for (int i = 0; i + 1 < n; ++i) {  // forward: node i and i+1
        const double c = 1.0 / (x[i + 1] - x[i]);
        Df[i * n + i] = -c;
        Df[i * n + i + 1] = c;
    }
    Df[n2 - 2] = -last; Df[n2 - 1] = last;  // last row: backward
    Db[0] = -first; Db[1] = first;          // first row: forward
    for (int i = 1; i < n; ++i) {  // backward: node i-1 and i
        const double c = 1.0 / (x[i] - x[i - 1]);
        Db[i * n + i - 1] = -c;
        Db[i * n + i] = c;
    }
    return ESDG_OK;
}

int esdg_basis(int N, int FluxDifferencing, double* xGL, double* wGL, double* xG, double* wG, double* D, double* D0,
               double* Dstrong, double* Dhat, double* VdmInv) {
    if (N < 1 || N > 15) return ESDG_E_ARG;
    esdg::Basis B;
    esdg::build_basis(N, FluxDifferencing, &B);
    const int n = N + 1;
    auto cp = [](double* dst, const std::vector<double>& v) { if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(double)); };
    cp(xGL, B.xGL); cp(wGL, B.wGL); cp(xG, B.xG); cp(wG, B.wG);
    cp(D, B.D); cp(D0, B.D0); cp(Dstrong, B.Dstrong); cp(Dhat, B.Dhat); cp(VdmInv, B.VdmInv);
    (void)n;
    return ESDG_OK;
}

int esdg_mesh_cartesian(int N, double xL, double xR, double yL, double yR, int NX, int NY, int periodic_rows,
                        int periodic_cols, esdg_mesh** out) {
    if (!out || N < 1 || N > 15 || NX < 1 || NY < 1) return ESDG_E_ARG;
    if ((periodic_rows && NY < 2) || (periodic_cols && NX < 2)) return ESDG_E_ARG;
    esdg_mesh* m = new (std::nothrow) esdg_mesh(N);
    if (!m) return ESDG_E_NOMEM;
    try {
        m->m.generate_cartesian(xL, xR, yL, yR, NX, NY, periodic_rows != 0, periodic_cols != 0);
    } catch (const std::exception& ex) {
        esdg::g_create_error = ex.what();
        delete m;
        return ESDG_E_ARG;
    }
    *out = m;
    return ESDG_OK;
}

int esdg_mesh_mapped(int N, double xL, double xR, double yL, double yR, int NX, int NY, double amp, int m_order,
                     unsigned rotate_seed, esdg_mesh** out) {
    if (!out || N < 1 || N > 15 || NX < 1 || NY < 1 || m_order < 1 || m_order > 32) return ESDG_E_ARG;
    esdg_mesh* m = new (std::nothrow) esdg_mesh(N);
    if (!m) return ESDG_E_NOMEM;
    try {
        m->m.generate_mapped(xL, xR, yL, yR, NX, NY, amp, m_order, rotate_seed);
    } catch (const std::exception& ex) {
        esdg::g_create_error = ex.what();
        delete m;
        return ESDG_E_ARG;
    }
    *out = m;
    return ESDG_OK;
}

int esdg_mesh_read_ism2(int N, const char* path, int read_bottom, int convert_km, esdg_mesh** out) {
    if (!out || !path || N < 1 || N > 15) return ESDG_E_ARG;
    esdg_mesh* m = new (std::nothrow) esdg_mesh(N);
    if (!m) return ESDG_E_NOMEM;
    try {
        m->m.read_ism2(path, read_bottom != 0, convert_km != 0);
    } catch (const std::exception& ex) {
        esdg::g_create_error = ex.what();
        delete m;
        return ESDG_E_IO;
    }
    *out = m;
    return ESDG_OK;
}

int esdg_mesh_write_ism2(const esdg_mesh* m, const char* path) {
    if (!m || !path) return ESDG_E_ARG;
    try {
        m->m.write_ism2(path);
    } catch (const std::exception& ex) {
        esdg::g_create_error = ex.what();
        return ESDG_E_IO;
    }
    return ESDG_OK;
}

int esdg_mesh_element_curves(const esdg_mesh* m, int* curve_order, double* corners, int* curved, double* curves) {
    if (!m || !curve_order) return ESDG_E_ARG;
    const esdg::Mesh& M = m->m;
    if (M.elem_corners.empty()) {
        esdg::g_create_error = "mesh_element_curves: the mesh has no corner lists (Cartesian meshes are generated without curves)";
        return ESDG_E_UNSUPPORTED;
    }
    const int mo = M.curve_order, mm = mo > 0 ? mo : 1;
    *curve_order = mm;
    if (!corners && !curved && !curves) return ESDG_OK;
    if (!corners || !curved || !curves) return ESDG_E_ARG;
    const int K = M.K, stride = M.elem_curves_stride ? M.elem_curves_stride : 2;
    for (int e = 0; e < K; ++e)
        for (int k = 0; k < 4; ++k) {
            const int nd = M.elem_corners[(size_t)e * 4 + k];
            corners[((size_t)e * 4 + k) * 2 + 0] = M.nodes_x[nd];
            corners[((size_t)e * 4 + k) * 2 + 1] = M.nodes_y[nd];
            const int c = M.elem_curved.empty() ? 0 : M.elem_curved[(size_t)e * 4 + k];
            curved[(size_t)e * 4 + k] = c;
            for (int j = 0; j <= mm; ++j) {
                double* o = &curves[(((size_t)e * 4 + k) * (mm + 1) + j) * 2];
                if (c && j <= mo) {
                    const double* v = &M.elem_curves[(((size_t)e * 4 + k) * (mo + 1) + j) * stride];
                    o[0] = v[0]; o[1] = v[1];
                } else {
                    o[0] = 0.0; o[1] = 0.0;
                }
            }
        }
    return ESDG_OK;
}

int esdg_geometry_device(int N, int K, int curve_order, const double* corners, const int* curved,
                         const double* curves, double* x, double* y, double* x_xi, double* x_eta, double* y_xi,
                         double* y_eta, double* J, double* nx_side, double* ny_side, double* scal_side, void* stream) {
    if (N < 1 || N > 7) { esdg::g_create_error = "geometry_device: N must be in 1..7"; return ESDG_E_UNSUPPORTED; }
    if (curve_order < 1 || curve_order > esdg::GEO_MAXM) {
        esdg::g_create_error = "geometry_device: curve order must be in 1.." + std::to_string(esdg::GEO_MAXM);
        return ESDG_E_UNSUPPORTED;
    }
    if (K <= 0 || !corners || !curved || !curves || !x || !y || !x_xi || !x_eta || !y_xi || !y_eta || !J ||
        !nx_side || !ny_side || !scal_side) {
        esdg::g_create_error = "geometry_device: K must be positive and every array given";
        return ESDG_E_ARG;
    }
    esdg::Basis B;
    esdg::build_basis(N, 1, &B);
    esdg::GeoConst G;
    std::memset(&G, 0, sizeof G);
    const int ngl = N + 1;
    for (int i = 0; i < ngl; ++i) G.xg[i] = B.xGL[i];
    for (int i = 0; i < ngl * ngl; ++i) G.D0[i] = B.D0[i];
    esdg::curve_nodes_weights(curve_order, G.xc, G.wb);
    G.tol = std::pow(10.0, -12);
    G.m = curve_order;
    esdg::GeoArgs a{K, corners, curved, curves, x, y, x_xi, x_eta, y_xi, y_eta, J, nx_side, ny_side, scal_side};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (ngl) {
#define ESDG_GEO(NG)                                                                                  \
    case NG: {                                                                                        \
        using S = esdg::GeoShape<NG>;                                                                 \
        esdg::k_geometry<NG><<<(K + S::NE - 1) / S::NE, S::THREADS, 0, s>>>(a, G);                    \
        break;                                                                                        \
    }
        ESDG_GEO(2) ESDG_GEO(3) ESDG_GEO(4) ESDG_GEO(5) ESDG_GEO(6) ESDG_GEO(7) ESDG_GEO(8)
#undef ESDG_GEO
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        esdg::g_create_error = std::string("geometry_device: ") + cudaGetErrorString(e);
        return ESDG_E_CUDA;
    }
    return ESDG_OK;
}

int esdg_okada_uplift(long long n, const double* x, const double* y, const double* fault, int mercator, int add,
                      double* out, void* stream) {
    if (n <= 0 || !x || !y || !fault || !out) {
        esdg::g_create_error = "okada_uplift: n must be positive and every array given";
        return ESDG_E_ARG;
    }
    // fault: x0, y0, depth, length, width, strike, rake, dip, slip
    const double x0 = fault[0], y0 = fault[1], depth = fault[2], length = fault[3], width = fault[4];
    const double strike = fault[5], rake = fault[6], dip = fault[7], slip = fault[8];
    if (!(width > 0.0) || !(length > 0.0)) {
        esdg::g_create_error = "okada_uplift: length and width must be positive";
        return ESDG_E_ARG;
    }
    esdg::OkadaConst c;
    std::memset(&c, 0, sizeof c);
    const double rad = M_PI / 180.0;
    const double ang_l = rad * dip, ang_r = rad * rake, ang_t = rad * strike;
    c.x0 = x0; c.y0 = y0;
    c.halfl = 0.5 * length; c.width = width;
    c.hh = depth + width * std::sin(ang_l);
    c.sn_l = std::sin(ang_l); c.cs_l = std::cos(ang_l);
    c.sn_t = std::sin(ang_t); c.cs_t = std::cos(ang_t);
    c.del_x = width * std::cos(ang_l) * std::cos(ang_t);
    c.del_y = width * std::cos(ang_l) * std::sin(ang_t);
    c.ds = slip * std::cos(ang_r); c.dd = slip * std::sin(ang_r);
    c.reach = 1.5 * std::max(length, width);
    c.R = 6.378e6; c.rad = rad;
    if (mercator) {
        const double x0m = x0 * c.R * M_PI / 180.0;
        const double y0m = c.R * std::asinh(std::tan(y0 / 180.0 * M_PI));
        c.xlower = x0m - length; c.xupper = x0m + length; c.ylower = y0m - width; c.yupper = y0m + width;
        c.xo = (c.xlower / c.R) * (180.0 / M_PI);
        c.yo = std::atan(std::sinh(c.ylower / c.R)) * (180.0 / M_PI);
        c.yl = c.R * (y0 - c.yo) * rad - c.del_y;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (mercator) esdg::k_okada<true><<<blocks, 256, 0, s>>>((long)n, x, y, c, out, add);
    else esdg::k_okada<false><<<blocks, 256, 0, s>>>((long)n, x, y, c, out, add);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        esdg::g_create_error = std::string("okada_uplift: ") + cudaGetErrorString(e);
        return ESDG_E_CUDA;
    }
    return ESDG_OK;
}

int esdg_mesh_sizes(const esdg_mesh* m, int* K, int* F) {
    if (!m) return ESDG_E_ARG;
    if (K) *K = m->m.K;
    if (F) *F = m->m.F;
    return ESDG_OK;
}

int esdg_mesh_pack(const esdg_mesh* m, double* x, double* y, double* x_xi, double* x_eta, double* y_xi,
                   double* y_eta, double* Jinv, double* nx, double* ny, double* scal, double* b, int* EdgeData,
                   int* EdgeReversed, int* ElemToEdge, int* ElemEdgeMasterSlave, int* ElemEdgeOrientation) {
    if (!m) return ESDG_E_ARG;
    esdg::PackedMesh P;
    m->m.pack(&P);
    auto cpd = [](double* dst, const std::vector<double>& v) { if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(double)); };
    auto cpi = [](int* dst, const std::vector<int>& v) { if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(int)); };
    cpd(x, P.x); cpd(y, P.y); cpd(x_xi, P.xXi); cpd(x_eta, P.xEta); cpd(y_xi, P.yXi); cpd(y_eta, P.yEta);
    cpd(Jinv, P.Jinv); cpd(nx, P.nx); cpd(ny, P.ny); cpd(scal, P.scal); cpd(b, P.b);
    cpi(EdgeData, P.EdgeData); cpi(EdgeReversed, P.EdgeReversed); cpi(ElemToEdge, P.ElemToEdge);
    cpi(ElemEdgeMasterSlave, P.MasterSlave); cpi(ElemEdgeOrientation, P.Orientation);
    return ESDG_OK;
}

void esdg_mesh_free(esdg_mesh* m) { delete m; }

int esdg_bottom_derivatives(int K, int N, const double* D0, const double* b, const double* y_eta, const double* y_xi,
                            const double* x_eta, const double* x_xi, const double* Jinv, double* Bx, double* By) {
    if (K <= 0 || N < 1 || !D0 || !b || !y_eta || !y_xi || !x_eta || !x_xi || !Jinv || !Bx || !By) return ESDG_E_ARG;
    esdg::bottom_derivatives(K, N + 1, D0, b, y_eta, y_xi, x_eta, x_xi, Jinv, Bx, By);
    return ESDG_OK;
}

int esdg_element_sizes(int K, int N, const double* wGL, const double* Jinv, double* EleSizes, double* minEleSize) {
    if (K <= 0 || N < 1 || !wGL || !Jinv || !EleSizes || !minEleSize) return ESDG_E_ARG;
    *minEleSize = esdg::element_sizes(K, N + 1, wGL, Jinv, EleSizes);
    return ESDG_OK;
}

int esdg_rk_coefficients(int order, int ssp, double* A, double* B, double* C, int* stages) {
    if (!A || !B || !C || !stages) return ESDG_E_ARG;
    const int s = esdg::rk_coefficients(order, ssp, A, B, C);
    if (s == 0) return ESDG_E_UNSUPPORTED;
    *stages = s;
    return ESDG_OK;
}

int esdg_diagnostics(int K, int N, const double* wGL, const double* Jinv, const double* q, const double* qref,
                     const double* b, double g, double* L2, double* Linf, double* mass, double* entropy) {
    if (K <= 0 || N < 1 || !wGL || !Jinv || !q) return ESDG_E_ARG;
    esdg::diagnostics(K, N + 1, wGL, Jinv, q, qref, b, g, L2, Linf, mass, entropy);
    return ESDG_OK;
}

}  // extern "C"

// ===========================================================================
// Right-hand side without any allocation (esdg_compute_rhs_noalloc).
//
// For callers that may not allocate device memory themselves: hosts whose
// memory is owned by their own pool allocator, and serving loops that must
// not stall on cudaMalloc/cudaFree (both synchronise the device).  They pass
// their own device buffers for the inputs and the output; the scratch this
// evaluation needs (packed face/side tables, bathymetry traces, face fluxes,
// a step state) lives in one file-scope device array of fixed size.  The
// call reads the count of bad connectivity entries back to the host and
// synchronises its stream before it returns.
// ===========================================================================
namespace esdg {

// 16 MiB of scratch per device, held from library load until process exit.
constexpr long long kNoAllocScratchDoubles = 1ll << 21;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

struct NoAllocLayout {
    long long st, err, ftab, side, bL, bR, SP, total;  // offsets in doubles
};

static NoAllocLayout noalloc_layout(int K, int F, int ngl) {
    auto up = [](long long v) { return (v + 31) / 32 * 32; };  // 256-byte segments
    NoAllocLayout L;
    long long o = 0;
    L.st = o; o = up(o + (long long)(sizeof(DevState) + 7) / 8);
    L.err = o; o = up(o + 1);
    L.ftab = o; o = up(o + 2ll * F);
    L.side = o; o = up(o + 8ll * K);
    L.bL = o; o = up(o + (long long)F * ngl);
    L.bR = o; o = up(o + (long long)F * ngl);
    L.SP = o; o = up(o + 3ll * F * ngl);
    L.total = o;
    return L;
}

// Packs EdgeData / ElemToEdge / MasterSlave / Orientation into the tables the
// flux and element kernels read, replacing every out-of-range entry by a safe
// one and counting it, resets the step state, and gathers the bathymetry
// traces (okl/GatherEdgeData/CollectEdgeData_Bottom.okl:16-134).
__global__ void k_noalloc_prepare(int K, int F, int ngl, const int* __restrict__ ED, const int* __restrict__ E2E,
                                  const int* __restrict__ MS, const int* __restrict__ OR, const double* __restrict__ b,
                                  int4* ftab, int4* side, double* bL, double* bR, DevState* st, int* err) {
    const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid == 0) {
        DevState z;
        memset(&z, 0, sizeof z);
        z.T = 1.0;
        *st = z;
    }
    if (gid < F) {
        const int* r = ED + gid * 8;
        int eL = r[0], eR = r[1], sL = r[2], sR = r[3], same = r[4] ? 1 : 0, cpuL = r[5], cpuR = r[6];
        int bad = 0;
        if (eL < 0 || eL >= K || sL < 0 || sL > 3 || cpuL != 0) { bad = 1; eL = 0; sL = 0; }
        if (cpuR == -1) eR = -1;
        else if (cpuR != 0 || eR < 0 || eR >= K || sR < 0 || sR > 3) { bad = 1; eR = -1; }
        if (eR < 0) sR = 0;
        if (bad) atomicAdd(err, 1);
        ftab[gid] = make_int4(eL, eR, sL | (sR << 2) | (same << 4), 0);
        const int n2 = ngl * ngl;
        for (int i = 0; i < ngl; ++i) {
            const double vl = b[(long)eL * n2 + trace_offset(sL, i, ngl)];
            bL[gid * ngl + i] = vl;
            bR[gid * ngl + i] = (eR >= 0) ? b[(long)eR * n2 + trace_offset(sR, i, ngl)] : vl;
        }
    }
    if (gid < 4l * K) {
        int fc = E2E[gid] - 1, ms = MS[gid], orr = OR[gid];
        int bad = 0;
        if (fc < 0 || fc >= F) { bad = 1; fc = 0; }
        if (ms != 1 && ms != -1) { bad = 1; ms = 1; }
        if (orr != 0 && orr != 1) { bad = 1; orr = 1; }
        if (bad) atomicAdd(err, 1);
        side[gid] = make_int4(fc, ms, orr, 0);
    }
}

template <int NGL>
static void noalloc_launch(int K, int F, int NumFlux, const PhysConst& c, const double* q, const double* Jinv,
                           const double* Yxi, const double* Yeta, const double* Xxi, const double* Xeta,
                           const double* Bx, const double* By, const double* D, const double* nx, const double* ny,
                           const double* scal, double* base, const NoAllocLayout& L, double* Qt, cudaStream_t s) {
    DevState* st = reinterpret_cast<DevState*>(base + L.st);
    FaceArgs fa{F, reinterpret_cast<const int4*>(base + L.ftab), q, nx, ny, scal, base + L.bL, base + L.bR,
                base + L.SP, nullptr, nullptr, nullptr, st, c};
    const long nfn = (long)F * NGL;
    const int fb = (int)((nfn + 255) / 256);
    // face-major fluxes with the side table (SIDEOUT / SIDEIN off): the
    // scratch layout of this entry point
    if (NumFlux == 0) k_face_flux<NGL, 0, false, false, false><<<fb, 256, 0, s>>>(fa);
    else if (NumFlux == 2) k_face_flux<NGL, 2, false, false, false><<<fb, 256, 0, s>>>(fa);
    else k_face_flux<NGL, 3, false, false, false><<<fb, 256, 0, s>>>(fa);
    ElemArgs ea;
    memset(&ea, 0, sizeof ea);
    ea.K = K; ea.Jinv = Jinv; ea.Yxi = Yxi; ea.Yeta = Yeta; ea.Xxi = Xxi; ea.Xeta = Xeta; ea.Bx = Bx; ea.By = By;
    ea.D = D; ea.SP = base + L.SP; ea.side = reinterpret_cast<const int4*>(base + L.side);
    ea.q = const_cast<double*>(q); ea.Qt = Qt; ea.st = st; ea.mode = 2; ea.c = c;
    using S = ElemShape<NGL>;
    k_element<NGL, false><<<(K + S::NE - 1) / S::NE, S::THREADS, 0, s>>>(ea);
}

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[64] = {nullptr};

}  // namespace esdg

extern "C" int esdg_compute_rhs_noalloc(int N, int K, int F, int NumFlux, int ES, double g_const, double PosPresTOL,
                                        const double* q, const double* Jinv, const double* y_xi, const double* y_eta,
                                        const double* x_xi, const double* x_eta, const double* Bx, const double* By,
                                        const double* b, const double* Dmat, const double* nx, const double* ny,
                                        const double* scal, const int* EdgeData, const int* ElemToEdge,
                                        const int* ElemEdgeMasterSlave, const int* ElemEdgeOrientation, double* Qt,
                                        void* stream) {
    using namespace esdg;
    if (N < 1 || N > 7) { g_create_error = "compute_rhs_noalloc: N must be in 1..7"; return ESDG_E_UNSUPPORTED; }
    if (NumFlux != 0 && NumFlux != 2 && NumFlux != 3) {
        g_create_error = "compute_rhs_noalloc: NumFlux must be 0, 2 or 3";
        return ESDG_E_UNSUPPORTED;
    }
    if (K <= 0 || F <= 0 || !q || !Jinv || !y_xi || !y_eta || !x_xi || !x_eta || !Bx || !By || !b || !Dmat || !nx ||
        !ny || !scal || !EdgeData || !ElemToEdge || !ElemEdgeMasterSlave || !ElemEdgeOrientation || !Qt) {
        g_create_error = "compute_rhs_noalloc: sizes must be positive and every array given";
        return ESDG_E_ARG;
    }
    const int ngl = N + 1;
    const NoAllocLayout L = noalloc_layout(K, F, ngl);
    if (L.total > kNoAllocScratchDoubles) {
        g_create_error = "compute_rhs_noalloc: mesh needs " + std::to_string(L.total) +
                         " doubles of scratch, the fixed maximum is " + std::to_string(kNoAllocScratchDoubles) +
                         " (2*Nfaces + 8*Nelem + 5*Nfaces*(N+1), tables rounded up to 256 bytes)";
        return ESDG_E_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        g_create_error = std::string("compute_rhs_noalloc: cudaGetDevice: ") + cudaGetErrorString(e);
        return ESDG_E_CUDA;
    }
    if (stream) {
        // the kernels run on `stream` against this device's scratch address
        int sdev = -1;
        e = cudaStreamGetDevice(static_cast<cudaStream_t>(stream), &sdev);
        if (e != cudaSuccess) {
            g_create_error = std::string("compute_rhs_noalloc: cudaStreamGetDevice: ") + cudaGetErrorString(e);
            return ESDG_E_ARG;
        }
        if (sdev != dev) {
            g_create_error = "compute_rhs_noalloc: the stream belongs to device " + std::to_string(sdev) +
                             ", the current device is " + std::to_string(dev) + "; make the stream's device current";
            return ESDG_E_ARG;
        }
    }
    double* base = nullptr;
    {
        // the device address of the scratch array, looked up once per device
        // (with that device current) on the first call
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                g_create_error = std::string("compute_rhs_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return ESDG_E_CUDA;
            }
            g_noalloc_ptr[dev] = static_cast<double*>(p);
        }
        base = g_noalloc_ptr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int* err = reinterpret_cast<int*>(base + L.err);
    e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e != cudaSuccess) { g_create_error = std::string("compute_rhs_noalloc: ") + cudaGetErrorString(e); return ESDG_E_CUDA; }
    const long np = std::max<long>(F, 4l * K);
    k_noalloc_prepare<<<(int)((np + 255) / 256), 256, 0, s>>>(
        K, F, ngl, EdgeData, ElemToEdge, ElemEdgeMasterSlave, ElemEdgeOrientation, b,
        reinterpret_cast<int4*>(base + L.ftab), reinterpret_cast<int4*>(base + L.side), base + L.bL, base + L.bR,
        reinterpret_cast<DevState*>(base + L.st), err);
    PhysConst c;
    c.g = g_const; c.half_g = 0.5 * g_const; c.fourth_g = 0.25 * g_const;
    c.geomFace = 1.0 / (2.0 / (N * (N + 1.0)));
    c.PosPresTOL = PosPresTOL; c.eps0 = 0; c.sigmaMin = 0; c.sigmaMax = 0; c.ZeroTOL = std::pow(10.0, -5); c.sensor_skip = 0.0; c.ES = ES;
    switch (ngl) {
        case 2: noalloc_launch<2>(K, F, NumFlux, c, q, Jinv, y_xi, y_eta, x_xi, x_eta, Bx, By, Dmat, nx, ny, scal, base, L, Qt, s); break;
        case 3: noalloc_launch<3>(K, F, NumFlux, c, q, Jinv, y_xi, y_eta, x_xi, x_eta, Bx, By, Dmat, nx, ny, scal, base, L, Qt, s); break;
        case 4: noalloc_launch<4>(K, F, NumFlux, c, q, Jinv, y_xi, y_eta, x_xi, x_eta, Bx, By, Dmat, nx, ny, scal, base, L, Qt, s); break;
        case 5: noalloc_launch<5>(K, F, NumFlux, c, q, Jinv, y_xi, y_eta, x_xi, x_eta, Bx, By, Dmat, nx, ny, scal, base, L, Qt, s); break;
        case 6: noalloc_launch<6>(K, F, NumFlux, c, q, Jinv, y_xi, y_eta, x_xi, x_eta, Bx, By, Dmat, nx, ny, scal, base, L, Qt, s); break;
        case 7: noalloc_launch<7>(K, F, NumFlux, c, q, Jinv, y_xi, y_eta, x_xi, x_eta, Bx, By, Dmat, nx, ny, scal, base, L, Qt, s); break;
        default: noalloc_launch<8>(K, F, NumFlux, c, q, Jinv, y_xi, y_eta, x_xi, x_eta, Bx, By, Dmat, nx, ny, scal, base, L, Qt, s); break;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) { g_create_error = std::string("compute_rhs_noalloc: launch: ") + cudaGetErrorString(e); return ESDG_E_CUDA; }
    int nerr = 0;
    e = cudaMemcpyAsync(&nerr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { g_create_error = std::string("compute_rhs_noalloc: ") + cudaGetErrorString(e); return ESDG_E_CUDA; }
    if (nerr) {
        g_create_error = "compute_rhs_noalloc: " + std::to_string(nerr) + " connectivity entries out of range";
        return ESDG_E_ARG;
    }
    return ESDG_OK;
}

#include "esdg_arena.cuh"
#include "esdg_mlp_abi.cuh"
