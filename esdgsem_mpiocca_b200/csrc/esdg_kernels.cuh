// Per-stage kernels of the ES-DGSEM engine (sm_100a, FP64).
//
// One RK stage of the plain path is two launches:
//   face_flux  : one thread per face node gathers the two traces straight
//                from q (wall ghost on boundary faces), evaluates the ES
//                Riemann flux once and writes the scaled flux F*[F][3][ngl];
//   element    : NE elements per block staged in shared memory; flux-
//                differencing volume integral, lifting of the four face
//                fluxes, low-storage (or SSP) RK update and, on the last
//                stage, the element wave-speed maximum for the next dt.
// With artificial viscosity (BR1 gradient + viscous terms) a stage is the
// sensor pass (esdg_indicator.cuh; at the step start and before stages > 0)
// and four launches: face_flux (+ gradient face flux), element_av1 (inviscid
// Qt and the lifted gradient), face_visc, element_av2 (viscous volume and
// lift + RK update).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "esdg_physics.cuh"
#include "esdg_partialdry.cuh"

namespace esdg {

enum : int { ST_OK = 0, ST_NONFINITE = 1 };

// Per-instance time-stepping state, resident in device memory so that a
// whole step runs without a host round trip (and can be graph-captured).
struct DevState {
    double t, dt, T, minEle, CFL, DFL;
    unsigned long long lam_key, visc_key;
    int steps, max_steps, done, status;
    // checkpoint pause (pause_on != 0): a step does not start once t >=
    // pause_at and at least one step ran since steps == resume_steps; the
    // host writes its outputs and resumes (the reference's plot checkpoints,
    // src/deviceclass.cpp:1143-1147, one per step)
    double pause_at;
    int pause_on, resume_steps;
};

// Element-side face fluxes (the SP buffer of the engine): for side s of
// element e, the scaled ES flux of that side's face at the side's own nodes
// j = 0..NGL-1 (the element's orientation of the side), already multiplied
// by -MasterSlave: SP[((e * 4 + s) * 3 + eq) * NGL + j].  The element then
// adds fs * Jinv, which is the reference's -ms * flux * Jinv
// (okl/DG/SurfaceKernel.okl:17-142) bit for bit (the sign flip is exact),
// and bulk-copies its tile's fluxes with the rest of the tile.
__host__ __device__ __forceinline__ long side_flux_at(int e, int side, int eq, int j, int ngl) {
    return ((long)(e * 4 + side) * 3 + eq) * ngl + j;
}

// Packed face record: x elemL, y elemR or -1, z sideL | sideR << 2 |
// sameOrient << 4, w the element-side flags the face kernel needs to write
// element-side fluxes: orientation of the left side (bit 0), its
// MasterSlave == -1 (bit 1), the same two for the right side (bits 2, 3).
__host__ __device__ __forceinline__ int face_side_flags(int orientL, int msL, int orientR, int msR) {
    return (orientL ? 1 : 0) | (msL < 0 ? 2 : 0) | (orientR ? 4 : 0) | (msR < 0 ? 8 : 0);
}

struct FaceArgs {
    int F;
    const int4* __restrict__ ftab;  // (elemL, elemR or -1, sideL | sideR<<2 | sameOrient<<4, side flags)
    const double* __restrict__ q;
    const double* __restrict__ nx;
    const double* __restrict__ ny;
    const double* __restrict__ scal;
    const double* __restrict__ bL;
    const double* __restrict__ bR;
    double* __restrict__ SP;   // element-side fluxes [K][4][3][ngl] (face-major [F][3][ngl] without SIDEOUT)
    double* __restrict__ SGX;  // [F][2][ngl] (AV only)
    double* __restrict__ SGY;
    const int* __restrict__ elem_inst;
    const DevState* __restrict__ st;
    PhysConst c;
    // active set (null: every face): gradient fluxes only where an adjacent
    // element is flagged
    const int* __restrict__ act = nullptr;
    // live extent (null: all): [0] elements, [1] faces below which every
    // live entity lies (the arena keeps it current between replays)
    const int* __restrict__ extent = nullptr;
    // Testcase 1 (conv = 1): exact outer states on boundary faces at the
    // stage time t + tfrac dt, from the nodal coordinates X, Y
    int conv = 0;
    double tfrac = 0.0;
    const double* __restrict__ X = nullptr;
    const double* __restrict__ Y = nullptr;
};

struct ElemArgs {
    int K;
    const double* __restrict__ Jinv;
    const double* __restrict__ Yxi;
    const double* __restrict__ Yeta;
    const double* __restrict__ Xxi;
    const double* __restrict__ Xeta;
    const double* __restrict__ Bx;
    const double* __restrict__ By;
    const double* __restrict__ B;
    const double* __restrict__ D;       // flux-differencing matrix [ngl][ngl]
    const double* __restrict__ Dhat;    // BR1 gradient matrix
    const double* __restrict__ Dstrong; // viscous volume matrix
    const double* __restrict__ Vinv;    // modal transform
    const double* __restrict__ SP;      // element-side face fluxes [K][4][3][ngl] (see side_flux_at)
    const double* __restrict__ SGX;     // gradient face fluxes [F][2][ngl]
    const double* __restrict__ SGY;
    const double* __restrict__ SPV;     // viscous face fluxes [F][2][ngl]
    const int4* __restrict__ side;      // per element side: (face, masterSlave, orientation, 0)
    double* q;
    double* __restrict__ gRK;
    double* __restrict__ Qt;
    const double* __restrict__ Qtmp;
    double* __restrict__ GX;            // [K][2][ngl][ngl]
    double* __restrict__ GY;
    double* __restrict__ VP;            // [K]
    const int* __restrict__ elem_inst;
    DevState* st;
    double rkA, rkB, rkC;
    int mode;        // 0: LS-RK update, 1: SSP update, 2: write Qt only
    int lam;         // 1: element wave speed max into st[inst].lam_key after the update
    PhysConst c;
    // Active set (null: none).  Plain element kernels write Qt instead of
    // updating flagged elements and append them to alist (count in
    // *acount); k_element_av2 and k_grad_list then run over alist only.
    const int* __restrict__ act = nullptr;
    int* alist = nullptr;
    int* acount = nullptr;
    const int* __restrict__ extent = nullptr;  // live extent, as in FaceArgs
    // Partial-dry treatment (null: off): per-element dry flag, nodal b, and
    // the central / forward / backward difference matrices [n*n].
    const int* __restrict__ dry = nullptr;
    const double* __restrict__ Bn = nullptr;
    const double* __restrict__ Dc = nullptr;
    const double* __restrict__ Dup = nullptr;
    const double* __restrict__ Ddn = nullptr;
    // Testcase 1 (conv = 1): the manufactured source at the stage time
    // t + tfrac dt from the nodal coordinates X, Y (b: B, its derivatives:
    // Bx, By)
    int conv = 0;
    double tfrac = 0.0;
    const double* __restrict__ X = nullptr;
    const double* __restrict__ Y = nullptr;
    // Bounded waits of the bulk-copy kernels: limit in clock cycles (0: the
    // default, about 2 s) and, for a test of the timeout path, a tile whose
    // copies are never issued (tile + 1; 0: none).  Zero-initialised
    // arguments leave both off.
    long long wait_limit = 0;
    int skip_tile = 0;
};

// r += the manufactured source of node xid (Testcase 1).
__device__ __forceinline__ void add_conv_source(const ElemArgs& a, const DevState& S, long xid, double Bx, double By,
                                                double& r0, double& r1, double& r2) {
    double s0, s1, s2;
    conv_source(a.c.g, a.X[xid], a.Y[xid], S.t + a.tfrac * S.dt, Bx, By, a.B[xid], s0, s1, s2);
    r0 += s0;
    r1 += s1;
    r2 += s2;
}

__device__ __forceinline__ int inst_of(const int* elem_inst, int e) { return elem_inst ? elem_inst[e] : 0; }

// ---------------------------------------------------------------------------
// Face kernel.
// ---------------------------------------------------------------------------
// One face node (gid = face * NGL + node) of the face kernel.
template <int NGL, int NUMFLUX, bool AV, bool SIDEOUT>
__device__ __forceinline__ void face_flux_node(const FaceArgs& a, long gid) {
    const int f = (int)(gid / NGL), i = (int)(gid % NGL);
    constexpr int N2 = NGL * NGL;
    const int4 t = a.ftab[f];
    // the face's own data does not depend on the table entry: requested
    // together with it, ahead of the instance check
    const long ex = (long)f * NGL + i;
    const double nx = a.nx[ex], ny = a.ny[ex], sc = a.scal[ex], bLx = a.bL[ex];
    const int eL = t.x, eR = t.y, sL = t.z & 3, sR = (t.z >> 2) & 3, same = (t.z >> 4) & 1;
    // the instance's done flag (behind the instance table in an arena) is
    // requested together with the traces, not before them: a face of a
    // finished instance reads valid memory and stores nothing
    const DevState& S = a.st[inst_of(a.elem_inst, eL)];
    const int ir = same ? i : NGL - 1 - i;
    const double* qe = a.q + (long)eL * 3 * N2;
    const int oL = trace_offset(sL, i, NGL);
    const double hL = qe[oL], huL = qe[oL + N2], hvL = qe[oL + 2 * N2];
    double hR, huR, hvR;      // right state at master node i (flux)
    double ghR, ghuR, ghvR;   // right state at node i in the right element's order (gradient)
    const bool grad = AV && (!a.act || a.act[eL] || (eR >= 0 && a.act[eR]));
    if (eR >= 0) {
        const double* qr = a.q + (long)eR * 3 * N2;
        const int o = trace_offset(sR, ir, NGL);
        hR = qr[o]; huR = qr[o + N2]; hvR = qr[o + 2 * N2];
        if (grad) {
            const int o2 = trace_offset(sR, i, NGL);
            ghR = qr[o2]; ghuR = qr[o2 + N2]; ghvR = qr[o2 + 2 * N2];
        }
    } else {
        // The reference stores the ghost of every face node in order and reads
        // it back at node ir (okl/GatherEdgeData/SolidWalls.okl:150-173).
        const long exr = (long)f * NGL + ir;
        const int o = trace_offset(sL, ir, NGL);
        if (a.conv) {  // okl/GatherEdgeData/Dirichlet_ConvTest.okl:112-119, read back the same way
            const long xo = (long)eL * N2 + o;
            conv_exact(a.X[xo], a.Y[xo], S.t + a.tfrac * S.dt, a.bL[exr], hR, huR, hvR);
        } else {
            wall_ghost(a.nx[exr], a.ny[exr], qe[o], qe[o + N2], qe[o + 2 * N2], hR, huR, hvR);
        }
        if (grad) { ghR = hL; ghuR = huL; ghvR = hvL; }
    }
    const double bRx = a.bR[(long)f * NGL + ir];
    if (S.done) return;
    double N0, N1, N2f;
    es_flux<NUMFLUX>(a.c, nx, ny, hL, huL, hvL, hR, huR, hvR, bLx, bRx, N0, N1, N2f);
    const double s = sc;
    const double v0 = s * a.c.geomFace * N0, v1 = s * a.c.geomFace * N1, v2 = s * a.c.geomFace * N2f;
    if (SIDEOUT) {
        // both sides' copies, each in its element's node order and signed
        // by -MasterSlave (side_flux_at)
        const int w = t.w;
        const int jL = (w & 1) ? i : NGL - 1 - i;
        double* pl = a.SP + side_flux_at(eL, sL, 0, jL, NGL);
        const bool nL = (w & 2) != 0;
        pl[0] = nL ? v0 : -v0; pl[NGL] = nL ? v1 : -v1; pl[2 * NGL] = nL ? v2 : -v2;
        if (eR >= 0) {
            const int jR = (w & 4) ? i : NGL - 1 - i;
            double* pr = a.SP + side_flux_at(eR, sR, 0, jR, NGL);
            const bool nR = (w & 8) != 0;
            pr[0] = nR ? v0 : -v0; pr[NGL] = nR ? v1 : -v1; pr[2 * NGL] = nR ? v2 : -v2;
        }
    } else {
        double* sp = a.SP + (long)f * 3 * NGL + i;
        sp[0] = v0;
        sp[NGL] = v1;
        sp[2 * NGL] = v2;
    }
    if (grad) {
        // okl/BR1_Gradient/calcNumFluxesGradient.okl:16-135 (the right trace
        // is taken in the right element's own order, as there).
        const double tol = a.c.PosPresTOL;
        const double iL = (hL > tol) ? 1.0 / hL : 0.0;
        const double iR = (ghR > tol) ? 1.0 / ghR : 0.0;
        const double uL = huL * iL, uR = ghuR * iR, vL = hvL * iL, vR = ghvR * iR;
        double* gx = a.SGX + (long)f * 2 * NGL + i;
        double* gy = a.SGY + (long)f * 2 * NGL + i;
        gx[0] = nx * s * a.c.geomFace * 0.5 * (uL + uR);
        gx[NGL] = nx * s * a.c.geomFace * 0.5 * (vL + vR);
        gy[0] = ny * s * a.c.geomFace * 0.5 * (uL + uR);
        gy[NGL] = ny * s * a.c.geomFace * 0.5 * (vL + vR);
    }
}

// STRIDE = false: one thread per face node (a single mesh's one-shot
// grid).  STRIDE = true: a resident grid strides over the face nodes below
// the live extent (an arena, whose face capacity can be far above its live
// faces); a separate instantiation, since the loop costs registers.
// SIDEOUT = true: element-side fluxes (the engine); false: the face-major
// [F][3][ngl] layout of the allocation-free entry point.
template <int NGL, int NUMFLUX, bool AV, bool STRIDE = false, bool SIDEOUT = true>
__global__ void __launch_bounds__(256, STRIDE ? 4 : 1) k_face_flux(FaceArgs a) {
    long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long all = (long)a.F * NGL;
    if (!STRIDE) {
        // Descending face order.  Face ids follow the element order (a face
        // is numbered by the first element that has it) and the element
        // kernels walk their tiles upwards, so the first faces taken here
        // read the traces the element kernel wrote last, and the fluxes
        // written last are those of the first tiles the next element kernel
        // reads: both still in L2.
        const long n = a.extent ? min(all, (long)a.extent[1] * NGL) : all;
        if (gid >= n) return;
        face_flux_node<NGL, NUMFLUX, AV, SIDEOUT>(a, n - 1 - gid);
    } else {
        const long n = a.extent ? min(all, (long)a.extent[1] * NGL) : all;
        for (; gid < n; gid += (long)gridDim.x * blockDim.x) face_flux_node<NGL, NUMFLUX, AV, SIDEOUT>(a, gid);
    }
}

// Viscous face flux from the lifted gradients of both elements
// (okl/BR1_Gradient/CollectEdgeDataGradient.okl:17-194 and
// okl/ViscoseParts/calcNumFluxesViscose.okl:17-107); zero on walls.
template <int NGL>
__device__ __forceinline__ void face_visc_node(long gid, const int4* __restrict__ ftab, const double* __restrict__ nxa,
                                               const double* __restrict__ nya, const double* __restrict__ scal,
                                               const double* __restrict__ GX, const double* __restrict__ GY,
                                               const double* __restrict__ VP, double* __restrict__ SPV,
                                               const int* __restrict__ elem_inst, const DevState* __restrict__ st,
                                               double geomFace, const int* __restrict__ act) {
    constexpr int N2 = NGL * NGL;
    const int f = (int)(gid / NGL), i = (int)(gid % NGL);
    const int4 t = ftab[f];
    const int eL = t.x, eR = t.y, sL = t.z & 3, sR = (t.z >> 2) & 3, same = (t.z >> 4) & 1;
    // the done flag (behind the instance table in an arena) and the active
    // flags are requested together
    const bool done = st[inst_of(elem_inst, eL)].done;
    const long ex = (long)f * NGL + i;
    double N0 = 0.0, N1 = 0.0;
    // Active set: only faces of flagged elements are read.  A face with a
    // non-flagged side has zero viscosity on both sides (a flagged
    // neighbour would have flagged it), so its flux is zero.
    bool need = true;
    if (act) {
        const bool aL = act[eL] != 0, aR = eR >= 0 && act[eR] != 0;
        if (!aL && !aR) return;
        need = aL && aR;
    }
    if (done) return;
    if (eR >= 0 && need) {
        const int inc = same ? i : NGL - 1 - i;
        const long oL = (long)eL * 2 * N2 + trace_offset(sL, i, NGL);
        const long oR = (long)eR * 2 * N2 + trace_offset(sR, inc, NGL);
        const double nx = nxa[ex], ny = nya[ex];
        const double f2L = nx * GX[oL] + ny * GY[oL], f2R = nx * GX[oR] + ny * GY[oR];
        const double f3L = nx * GX[oL + N2] + ny * GY[oL + N2];
        const double f3R = nx * GX[oR + N2] + ny * GY[oR + N2];
        const double vm = fmax(VP[eL], VP[eR]);
        N0 = 0.5 * vm * (f2L + f2R);
        N1 = 0.5 * vm * (f3L + f3R);
    }
    const double s = scal[ex];
    SPV[(long)f * 2 * NGL + i] = -s * geomFace * N0;
    SPV[(long)f * 2 * NGL + NGL + i] = -s * geomFace * N1;
}

// One-shot or grid-stride over the face nodes (as k_face_flux).
template <int NGL, bool STRIDE = false>
__global__ void __launch_bounds__(256, STRIDE ? 4 : 1) k_face_visc(int F, const int4* __restrict__ ftab, const double* __restrict__ nxa,
                                                   const double* __restrict__ nya, const double* __restrict__ scal,
                                                   const double* __restrict__ GX, const double* __restrict__ GY,
                                                   const double* __restrict__ VP, double* __restrict__ SPV,
                                                   const int* __restrict__ elem_inst, const DevState* __restrict__ st,
                                                   double geomFace, const int* __restrict__ act = nullptr,
                                                   const int* __restrict__ extent = nullptr) {
    long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long all = (long)F * NGL;
    if (!STRIDE) {
        if (gid >= all || (extent && gid >= (long)extent[1] * NGL)) return;
        face_visc_node<NGL>(gid, ftab, nxa, nya, scal, GX, GY, VP, SPV, elem_inst, st, geomFace, act);
    } else {
        const long n = extent ? min(all, (long)extent[1] * NGL) : all;
        for (; gid < n; gid += (long)gridDim.x * blockDim.x)
            face_visc_node<NGL>(gid, ftab, nxa, nya, scal, GX, GY, VP, SPV, elem_inst, st, geomFace, act);
    }
}

// The viscous face fluxes of the active set only: the faces of the listed
// (flagged) elements alist[0 .. *acount), one thread per face node, grid
// stride.  A face of a listed element e is evaluated by e when e is its
// master side or when its master side is not flagged (then not listed), so
// each such face is evaluated exactly once, by face_visc_node (the same
// arithmetic as k_face_visc); faces with no flagged side are read by no
// one and left alone, as k_face_visc leaves them.  One thread per node of
// the listed elements' sides instead of one per face node of the mesh.
template <int NGL>
__global__ void __launch_bounds__(256) k_face_visc_list(const int4* __restrict__ side, const int4* __restrict__ ftab,
                                                        const double* __restrict__ nxa, const double* __restrict__ nya,
                                                        const double* __restrict__ scal, const double* __restrict__ GX,
                                                        const double* __restrict__ GY, const double* __restrict__ VP,
                                                        double* __restrict__ SPV, const int* __restrict__ elem_inst,
                                                        const DevState* __restrict__ st, double geomFace,
                                                        const int* __restrict__ act, const int* __restrict__ alist,
                                                        const int* __restrict__ acount) {
    const long n = (long)(*acount) * 4 * NGL;
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const int e = alist[k / (4 * NGL)];
        const int sd = (int)((k / NGL) % 4), i = (int)(k % NGL);
        const int f = side[(long)e * 4 + sd].x;
        const int4 t = ftab[f];
        // the master side evaluates the face (an element that is both sides
        // of a face, on a periodic strip, through its master side only);
        // the slave side only when the master is not flagged
        if (t.x == e ? sd != (t.z & 3) : act[t.x] != 0) continue;
        face_visc_node<NGL>((long)f * NGL + i, ftab, nxa, nya, scal, GX, GY, VP, SPV, elem_inst, st, geomFace, act);
    }
}

// ---------------------------------------------------------------------------
// Element kernels.
// ---------------------------------------------------------------------------
template <int NGL>
struct ElemShape {
    static constexpr int N2 = NGL * NGL;
    static constexpr int NE = (256 / N2) > 0 ? (256 / N2) : 1;  // elements per block
    static constexpr int THREADS = NE * N2;
};

// Wave-speed maximum folded into the owning instance's key
// (okl/DG/FindLambdaMax.okl:17-100 per node; a max, so the reduction order
// does not matter).  Warp-level and barrier-free: a shuffle reduction and
// one atomic per warp when all its lanes belong to one instance (always for
// a single mesh), one atomic per lane otherwise.  Must be called by every
// thread of the block (THREADS threads, the last warp possibly partial).
template <int THREADS>
__device__ __forceinline__ void warp_lambda(double lam, bool valid, int ins, DevState* st) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nl = (warp == (THREADS - 1) / 32 && (THREADS % 32) != 0) ? (THREADS % 32) : 32;
    const unsigned mask = (nl == 32) ? 0xffffffffu : ((1u << nl) - 1u);
    const int my = valid ? ins : -1;
    const int top = __reduce_max_sync(mask, my);
    if (top < 0) return;  // no valid lane in this warp
    const int low = -__reduce_max_sync(mask, valid ? -ins : -0x7fffffff);
    if (low == top) {
        double v = valid ? lam : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(mask, v, off);
            if (lane + off < nl) v = (isnan(o) || o > v) ? o : v;
        }
        if (lane == 0) atomicMax(&st[top].lam_key, dbl_key(v));
    } else if (valid) {
        atomicMax(&st[ins].lam_key, dbl_key(lam));
    }
}

__device__ __forceinline__ double node_lambda(const PhysConst& c, double h, double hu, double hv) {
    const double inv = (h > c.PosPresTOL) ? 1.0 / h : 0.0;
    const double cc = sqrt(c.g * h);
    return cc + fmax(fabs(hu * inv), fabs(hv * inv));
}

// Flux-differencing volume term + surface lift (+ RK update).
// okl/DG/VolumeKernelFluxDiffV99.okl:60-218, okl/DG/SurfaceKernel.okl:17-142,
// okl/RungeKutta/rkLS.okl:17-89 + UpdateKernelLS.okl:17-78 (mode 0),
// okl/RungeKutta/UpdateKernelSSP_V1.okl:17-98 (mode 1).
// SIDEIN = true: element-side fluxes (the engine); false: face-major fluxes
// with the side table (the allocation-free entry point).
template <int NGL, bool SIDEIN = true>
__global__ void __launch_bounds__(ElemShape<NGL>::THREADS) k_element(ElemArgs a) {
    constexpr int N2 = NGL * NGL, NE = ElemShape<NGL>::NE;
    __shared__ double sD[N2];
    __shared__ double sh[NE * N2], shu[NE * N2], shv[NE * N2], si[NE * N2];
    __shared__ double sYe[NE * N2], sYx[NE * N2], sXe[NE * N2], sXx[NE * N2];
    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    const int e0 = blockIdx.x * NE;
    if (a.extent && e0 >= a.extent[0]) return;  // whole block past the live extent
    const int e = e0 + el;
    const bool inb = e < a.K;
    const int ins = inb ? inst_of(a.elem_inst, e) : 0;
    const bool active = inb && !a.st[ins].done;
    const int xi = nd % NGL, eta = nd / NGL;
    if (tid < N2) sD[tid] = a.D[tid];
    const long xid = (long)e * N2 + nd, qid = (long)e * 3 * N2 + nd;
    const int s = el * N2 + nd;
    // Every global read of this thread is issued here, before the barrier,
    // so that their latencies overlap: state and metrics (staged for the
    // partners), Jinv/Bx/By, gRK (or Qtmp) and the face fluxes of the
    // node's sides.
    double h = 0, hu = 0, hv = 0, J = 0, bx = 0, by = 0, o0 = 0, o1 = 0, o2 = 0, dt = 0;
    double f[2][3] = {{0, 0, 0}, {0, 0, 0}};  // signed side fluxes, -ms * flux
    bool has[2] = {false, false};
    const bool to_list = active && a.act && a.act[e] != 0;
    if (active) {
        h = a.q[qid]; hu = a.q[qid + N2]; hv = a.q[qid + 2 * N2];
        sh[s] = h; shu[s] = hu; shv[s] = hv;
        sYe[s] = a.Yeta[xid]; sYx[s] = a.Yxi[xid]; sXe[s] = a.Xeta[xid]; sXx[s] = a.Xxi[xid];
        J = a.Jinv[xid]; bx = a.Bx[xid]; by = a.By[xid];
        if (a.mode == 0) { o0 = a.gRK[qid]; o1 = a.gRK[qid + N2]; o2 = a.gRK[qid + 2 * N2]; }
        else if (a.mode == 1) { o0 = a.Qtmp[qid]; o1 = a.Qtmp[qid + N2]; o2 = a.Qtmp[qid + 2 * N2]; }
        if (a.mode != 2) dt = a.st[ins].dt;
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            int side = -1, j = 0;
            if (pass == 0) {
                if (eta == 0) { side = 0; j = xi; }
                else if (eta == NGL - 1) { side = 2; j = xi; }
            } else {
                if (xi == NGL - 1) { side = 1; j = eta; }
                else if (xi == 0) { side = 3; j = eta; }
            }
            if (side >= 0) {
                has[pass] = true;
                if (SIDEIN) {
                    const double* fp = a.SP + side_flux_at(e, side, 0, j, NGL);
                    f[pass][0] = fp[0]; f[pass][1] = fp[NGL]; f[pass][2] = fp[2 * NGL];
                } else {
                    const int4 sd = a.side[(long)e * 4 + side];
                    const int inc = sd.z ? j : NGL - 1 - j;
                    const double* fp = a.SP + (long)sd.x * 3 * NGL + inc;
                    const double m = -sd.y;
                    f[pass][0] = m * fp[0]; f[pass][1] = m * fp[NGL]; f[pass][2] = m * fp[2 * NGL];
                }
            }
        }
        si[s] = (h > 0) ? 1.0 / h : 0.0;
    }
    __syncthreads();
    double lam = 0.0;
    if (active) {
        const int rb = el * N2 + eta * NGL;  // row base (same eta)
        const int cb = el * N2 + xi;         // column base (same xi)
        const double ih = si[s], ye = sYe[s], yx = sYx[s], xe = sXe[s], xx = sXx[s];
        const double fg = a.c.fourth_g, hg = a.c.half_g;
        double d1 = 0.0, d2 = 0.0, d3 = 0.0;
#pragma unroll
        for (int l = 0; l < NGL; ++l) {
            const int p = rb + l;
            const double dl = sD[xi * NGL + l];
            double f1, f2, f3;
            two_point_xi(fg, hg, h, hu, hv, ih, sh[p], shu[p], shv[p], si[p], ye, sYe[p], xe, sXe[p], f1, f2, f3);
            d1 += dl * f1; d2 += dl * f2; d3 += dl * f3;
        }
#pragma unroll
        for (int l = 0; l < NGL; ++l) {
            const int p = cb + l * NGL;
            const double dl = sD[eta * NGL + l];
            double g1, g2, g3;
            two_point_eta(fg, hg, h, hu, hv, ih, sh[p], shu[p], shv[p], si[p], yx, sYx[p], xx, sXx[p], g1, g2, g3);
            d1 += dl * g1; d2 += dl * g2; d3 += dl * g3;
        }
        double r0 = -J * d1;
        double r1 = -J * d2 - a.c.g * h * bx;
        double r2 = -J * d3 - a.c.g * h * by;
        if (a.dry && a.dry[e])
            pd_volume<NGL>(a.c, a.Dc, a.Dup, a.Ddn, sh + el * N2, a.Bn + (long)e * N2, eta, xi, ye, yx, xe, xx, J, r1,
                           r2);
        // lift: sides 0/2 first, then 1/3 (DBSurf1/2 are zero)
        const double db = 0.0;
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            if (has[pass]) {
                r0 += f[pass][0] * J;
                r1 += J * f[pass][1] + J * db;
                r2 += J * f[pass][2] + J * db;
            }
        }
        if (a.conv) add_conv_source(a, a.st[ins], xid, bx, by, r0, r1, r2);
        if (a.mode == 2 || to_list) {
            a.Qt[qid] = r0; a.Qt[qid + N2] = r1; a.Qt[qid + 2 * N2] = r2;
            if (to_list && nd == 0) a.alist[atomicAdd(a.acount, 1)] = e;
        } else {
            double q0, q1, q2;
            if (a.mode == 0) {
                const double g0 = a.rkA * o0 + r0;
                const double g1 = a.rkA * o1 + r1;
                const double g2 = a.rkA * o2 + r2;
                a.gRK[qid] = g0; a.gRK[qid + N2] = g1; a.gRK[qid + 2 * N2] = g2;
                q0 = h + a.rkC * dt * g0;
                q1 = hu + a.rkC * dt * g1;
                q2 = hv + a.rkC * dt * g2;
            } else {
                q0 = a.rkA * o0 + a.rkB * h + a.rkC * dt * r0;
                q1 = a.rkA * o1 + a.rkB * hu + a.rkC * dt * r1;
                q2 = a.rkA * o2 + a.rkB * hv + a.rkC * dt * r2;
            }
            a.q[qid] = q0; a.q[qid + N2] = q1; a.q[qid + 2 * N2] = q2;
            if (a.lam) lam = node_lambda(a.c, q0, q1, q2);
        }
    }
    if (a.lam) warp_lambda<ElemShape<NGL>::THREADS>(lam, active && !to_list, ins, a.st);
}

// Tail of the modal energy sensor (okl/ShockCapturing/ShockCapturing.okl:131-227):
// energy ratios of the highest modes from the modal coefficients w
// [mode_xi][mode_eta], log10, and the sine ramp between sigma_min and
// sigma_max.  Sums in the reference's order.
template <int NGL>
__device__ double sensor_tail(const PhysConst& c, const double* w) {
    constexpr int N = NGL - 1;
    double z1 = 0, n1 = 0, z2 = 0, n2s = 0;
    for (int i = 0; i < N; ++i) z1 += w[i * NGL + N] * w[i * NGL + N] + w[N * NGL + i] * w[N * NGL + i];
    z1 += w[N * NGL + N] * w[N * NGL + N];
    for (int i = 0; i < N - 1; ++i)
        z2 += w[i * NGL + N - 1] * w[i * NGL + N - 1] + w[(N - 1) * NGL + i] * w[(N - 1) * NGL + i];
    z2 += w[(N - 1) * NGL + N - 1] * w[(N - 1) * NGL + N - 1];
    for (int i = 0; i < NGL; ++i)
        for (int j = 0; j < NGL; ++j) n1 += w[i * NGL + j] * w[i * NGL + j];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) n2s += w[i * NGL + j] * w[i * NGL + j];
    const double t1 = (n1 < c.ZeroTOL) ? 0.0 : z1 / n1;
    const double t2 = (n1 < c.ZeroTOL) ? 0.0 : z2 / n2s;
    const double ratio = (t1 < t2) ? t2 : t1;
    // exact shortcut: log10 is accurate to an ulp, so below this bound the
    // reference's test sigmaMin >= log10(ratio) holds (NaN falls through)
    if (ratio < c.sensor_skip) return 0.0;
    const double sig = log10(ratio);
    if (c.sigmaMin >= sig) return 0.0;
    if (c.sigmaMax >= sig) {
        const double delta = 1.0 + sin(M_PI * (sig - 0.5 * (c.sigmaMax + c.sigmaMin)) / (c.sigmaMax - c.sigmaMin));
        return c.eps0 * 0.5 * delta;
    }
    return c.eps0;
}

// Modal transform entries of the sensor: M1[i][j] = sum_l V[i][l] m[j][l]
// and w[i][j] = sum_l M1[i][l] V[j][l] (s_Q1modal[i][j] of the reference
// holds node (xi=i, eta=j)); one entry per call, so that a thread per entry
// computes exactly what the serial loops do.
template <int NGL>
__device__ __forceinline__ double sensor_m1(const double* V, const double* m, int i, int j) {
    double acc = 0.0;
    for (int l = 0; l < NGL; ++l) acc += V[i * NGL + l] * m[j * NGL + l];
    return acc;
}
template <int NGL>
__device__ __forceinline__ double sensor_w(const double* V, const double* M1, int i, int j) {
    double acc = 0.0;
    for (int l = 0; l < NGL; ++l) acc += M1[i * NGL + l] * V[j * NGL + l];
    return acc;
}

// Inviscid volume + lift written to Qt and the
// lifted, h-scaled BR1 gradient of the velocities.
// okl/BR1_Gradient/calcGradient.okl:18-156, SurfaceKernelGradient.okl:16-150,
// scaleGradient.okl:17-60.
template <int NGL>
__global__ void __launch_bounds__(ElemShape<NGL>::THREADS) k_element_av1(ElemArgs a) {
    constexpr int N2 = NGL * NGL, NE = ElemShape<NGL>::NE;
    __shared__ double sD[N2], sDh[N2], sV[N2];
    __shared__ double sh[NE * N2], shu[NE * N2], shv[NE * N2], si[NE * N2];
    __shared__ double sYe[NE * N2], sYx[NE * N2], sXe[NE * N2], sXx[NE * N2];
    __shared__ double su[NE * N2], sv[NE * N2];
    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    const int e0 = blockIdx.x * NE;
    const int e = e0 + el;
    const bool inb = e < a.K;
    const int ins = inb ? inst_of(a.elem_inst, e) : 0;
    const bool active = inb && !a.st[ins].done;
    if (tid < N2) {
        sD[tid] = a.D[tid];
        sDh[tid] = a.Dhat[tid];
        sV[tid] = a.Vinv[tid];
    }
    const long xid = (long)e * N2 + nd, qid = (long)e * 3 * N2 + nd;
    const int s = el * N2 + nd;
    double h = 0, hu = 0, hv = 0;
    if (active) {
        h = a.q[qid]; hu = a.q[qid + N2]; hv = a.q[qid + 2 * N2];
        sh[s] = h; shu[s] = hu; shv[s] = hv;
        si[s] = (h > 0) ? 1.0 / h : 0.0;
        const double iv = (h > a.c.PosPresTOL) ? 1.0 / h : 0.0;
        su[s] = hu * iv; sv[s] = hv * iv;
        sYe[s] = a.Yeta[xid]; sYx[s] = a.Yxi[xid]; sXe[s] = a.Xeta[xid]; sXx[s] = a.Xxi[xid];
    }
    __syncthreads();
    if (!active) return;  // no further block-wide synchronisation below
    const int xi = nd % NGL, eta = nd / NGL;
    const double J = a.Jinv[xid];
    {
        const int rb = el * N2 + eta * NGL, cb = el * N2 + xi;
        const double ih = si[s], ye = sYe[s], yx = sYx[s], xe = sXe[s], xx = sXx[s];
        const double fg = a.c.fourth_g, hg = a.c.half_g;
        double d1 = 0.0, d2 = 0.0, d3 = 0.0;
#pragma unroll
        for (int l = 0; l < NGL; ++l) {
            const int p = rb + l;
            const double dl = sD[xi * NGL + l];
            double f1, f2, f3;
            two_point_xi(fg, hg, h, hu, hv, ih, sh[p], shu[p], shv[p], si[p], ye, sYe[p], xe, sXe[p], f1, f2, f3);
            d1 += dl * f1; d2 += dl * f2; d3 += dl * f3;
        }
#pragma unroll
        for (int l = 0; l < NGL; ++l) {
            const int p = cb + l * NGL;
            const double dl = sD[eta * NGL + l];
            double g1, g2, g3;
            two_point_eta(fg, hg, h, hu, hv, ih, sh[p], shu[p], shv[p], si[p], yx, sYx[p], xx, sXx[p], g1, g2, g3);
            d1 += dl * g1; d2 += dl * g2; d3 += dl * g3;
        }
        double r0 = -J * d1;
        double r1 = -J * d2 - a.c.g * h * a.Bx[xid];
        double r2 = -J * d3 - a.c.g * h * a.By[xid];
        if (a.dry && a.dry[e])
            pd_volume<NGL>(a.c, a.Dc, a.Dup, a.Ddn, sh + el * N2, a.Bn + (long)e * N2, eta, xi, ye, yx, xe, xx, J, r1,
                           r2);
        double gx0 = 0, gx1 = 0, gy0 = 0, gy1 = 0;
        {
            // calcGradient: u_xi = sum_l Dhat[xi][l] u(l,eta), u_eta = sum_l Dhat[eta][l] u(xi,l)
            double uxi = 0, ueta = 0, vxi = 0, veta = 0;
#pragma unroll
            for (int l = 0; l < NGL; ++l) {
                uxi += sDh[xi * NGL + l] * su[rb + l];
                ueta += sDh[eta * NGL + l] * su[cb + l * NGL];
                vxi += sDh[xi * NGL + l] * sv[rb + l];
                veta += sDh[eta * NGL + l] * sv[cb + l * NGL];
            }
            const double ux = ye * uxi - yx * ueta, vx = ye * vxi - yx * veta;
            const double uy = -xe * uxi + xx * ueta, vy = -xe * vxi + xx * veta;
            gx0 = J * ux; gx1 = J * vx; gy0 = J * uy; gy1 = J * vy;
        }
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            int side = -1, j = 0;
            if (pass == 0) {
                if (eta == 0) { side = 0; j = xi; }
                else if (eta == NGL - 1) { side = 2; j = xi; }
            } else {
                if (xi == NGL - 1) { side = 1; j = eta; }
                else if (xi == 0) { side = 3; j = eta; }
            }
            if (side >= 0) {
                const int4 sd = a.side[(long)e * 4 + side];
                const int inc = sd.z ? j : NGL - 1 - j;
                const double* fp = a.SP + side_flux_at(e, side, 0, j, NGL);
                const int ms = sd.y;
                const double db = 0.0;
                r0 += fp[0] * J;
                r1 += J * fp[NGL] + J * db;
                r2 += J * fp[2 * NGL] + J * db;
                const double* ux = a.SGX + (long)sd.x * 2 * NGL + inc;
                const double* uy = a.SGY + (long)sd.x * 2 * NGL + inc;
                if (pass == 0) gx0 += ms * ux[0] * J;
                else gx0 += ms * J * ux[0];
                gx1 += ms * J * ux[NGL];
                gy0 += ms * J * uy[0];
                gy1 += ms * J * uy[NGL];
            }
        }
        a.Qt[qid] = r0; a.Qt[qid + N2] = r1; a.Qt[qid + 2 * N2] = r2;
        const long gid = (long)e * 2 * N2 + nd;
        a.GX[gid] = h * gx0; a.GX[gid + N2] = h * gx1;
        a.GY[gid] = h * gy0; a.GY[gid + N2] = h * gy1;
    }
}

// Viscous volume term + viscous lift added to Qt, then the RK update, for
// the block's NE elements e0 + el (inb: element exists).
// okl/ViscoseParts/VolumeKernelViscose.okl:17-150, SurfaceKernelVisc.okl:17-144.
template <int NGL>
__device__ __forceinline__ void av2_tile(const ElemArgs& a, int e, bool inb, double* sDs, double* sF2, double* sF3,
                                         double* sG2, double* sG3) {
    constexpr int N2 = NGL * NGL;
    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    const int ins = inb ? inst_of(a.elem_inst, e) : 0;
    const bool active = inb && !a.st[ins].done;
    const long xid = (long)e * N2 + nd, qid = (long)e * 3 * N2 + nd, gid = (long)e * 2 * N2 + nd;
    const int s = el * N2 + nd;
    if (active) {
        const double eps = a.VP[e];
        const double F2 = eps * a.GX[gid], F3 = eps * a.GX[gid + N2];
        const double G2 = eps * a.GY[gid], G3 = eps * a.GY[gid + N2];
        const double ye = a.Yeta[xid], yx = a.Yxi[xid], xe = a.Xeta[xid], xx = a.Xxi[xid];
        sF2[s] = ye * F2 - xe * G2;
        sG2[s] = -yx * F2 + xx * G2;
        sF3[s] = ye * F3 - xe * G3;
        sG3[s] = -yx * F3 + xx * G3;
    }
    __syncthreads();
    double lam = 0.0;
    if (active) {
        const int xi = nd % NGL, eta = nd / NGL;
        const int rb = el * N2 + eta * NGL, cb = el * N2 + xi;
        double d2 = 0, d3 = 0;
#pragma unroll
        for (int l = 0; l < NGL; ++l) {
            d2 += sDs[xi * NGL + l] * sF2[rb + l];
            d2 += sDs[eta * NGL + l] * sG2[cb + l * NGL];
            d3 += sDs[xi * NGL + l] * sF3[rb + l];
            d3 += sDs[eta * NGL + l] * sG3[cb + l * NGL];
        }
        const double J = a.Jinv[xid];
        double r0 = a.Qt[qid], r1 = a.Qt[qid + N2], r2 = a.Qt[qid + 2 * N2];
        r1 += J * d2;
        r2 += J * d3;
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            int side = -1, j = 0;
            if (pass == 0) {
                if (eta == 0) { side = 0; j = xi; }
                else if (eta == NGL - 1) { side = 2; j = xi; }
            } else {
                if (xi == NGL - 1) { side = 1; j = eta; }
                else if (xi == 0) { side = 3; j = eta; }
            }
            if (side >= 0) {
                const int4 sd = a.side[(long)e * 4 + side];
                const int inc = sd.z ? j : NGL - 1 - j;
                const double* fp = a.SPV + (long)sd.x * 2 * NGL + inc;
                const int ms = sd.y;
                r1 += -ms * J * fp[0];
                r2 += -ms * J * fp[NGL];
            }
        }
        const double h = a.q[qid], hu = a.q[qid + N2], hv = a.q[qid + 2 * N2];
        if (a.mode == 2) {
            a.Qt[qid] = r0; a.Qt[qid + N2] = r1; a.Qt[qid + 2 * N2] = r2;
        } else {
            const double dt = a.st[ins].dt;
            double q0, q1, q2;
            if (a.mode == 0) {
                const double g0 = a.rkA * a.gRK[qid] + r0;
                const double g1 = a.rkA * a.gRK[qid + N2] + r1;
                const double g2 = a.rkA * a.gRK[qid + 2 * N2] + r2;
                a.gRK[qid] = g0; a.gRK[qid + N2] = g1; a.gRK[qid + 2 * N2] = g2;
                q0 = h + a.rkC * dt * g0;
                q1 = hu + a.rkC * dt * g1;
                q2 = hv + a.rkC * dt * g2;
            } else {
                q0 = a.rkA * a.Qtmp[qid] + a.rkB * h + a.rkC * dt * r0;
                q1 = a.rkA * a.Qtmp[qid + N2] + a.rkB * hu + a.rkC * dt * r1;
                q2 = a.rkA * a.Qtmp[qid + 2 * N2] + a.rkB * hv + a.rkC * dt * r2;
            }
            a.q[qid] = q0; a.q[qid + N2] = q1; a.q[qid + 2 * N2] = q2;
            if (a.lam) lam = node_lambda(a.c, q0, q1, q2);
        }
    }
    if (a.lam) warp_lambda<ElemShape<NGL>::THREADS>(lam, active, ins, a.st);
}

// Every element (alist null), or the elements of alist[0 .. *acount) with
// a grid-stride loop over tiles of NE list entries.
template <int NGL>
__global__ void __launch_bounds__(ElemShape<NGL>::THREADS) k_element_av2(ElemArgs a) {
    constexpr int N2 = NGL * NGL, NE = ElemShape<NGL>::NE;
    __shared__ double sDs[N2];
    __shared__ double sF2[NE * N2], sF3[NE * N2], sG2[NE * N2], sG3[NE * N2];
    const int tid = threadIdx.x;
    const int el = tid / N2;
    if (tid < N2) sDs[tid] = a.Dstrong[tid];
    if (!a.alist) {
        const int e = blockIdx.x * NE + el;
        av2_tile<NGL>(a, e, e < a.K, sDs, sF2, sF3, sG2, sG3);
        return;
    }
    const int count = *a.acount;
    for (int t = blockIdx.x; t * NE < count; t += gridDim.x) {
        const int idx = t * NE + el;
        const bool inb = idx < count;
        av2_tile<NGL>(a, inb ? a.alist[idx] : 0, inb, sDs, sF2, sF3, sG2, sG3);
        __syncthreads();  // shared tiles are rewritten by the next iteration
    }
}

// BR1 gradient (lifted, h-scaled) of the elements of alist[0 .. *acount):
// the gradient part of k_element_av1, in the same arithmetic order.
// okl/BR1_Gradient/calcGradient.okl:18-156, SurfaceKernelGradient.okl:16-150,
// scaleGradient.okl:17-60.
template <int NGL>
__global__ void __launch_bounds__(ElemShape<NGL>::THREADS) k_grad_list(ElemArgs a) {
    constexpr int N2 = NGL * NGL, NE = ElemShape<NGL>::NE;
    __shared__ double sDh[N2];
    __shared__ double su[NE * N2], sv[NE * N2];
    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    const int xi = nd % NGL, eta = nd / NGL;
    if (tid < N2) sDh[tid] = a.Dhat[tid];
    const int count = *a.acount;
    for (int t = blockIdx.x; t * NE < count; t += gridDim.x) {
        const int idx = t * NE + el;
        const bool inb = idx < count;
        const int e = inb ? a.alist[idx] : 0;
        const long xid = (long)e * N2 + nd, qid = (long)e * 3 * N2 + nd;
        const int s = el * N2 + nd;
        double h = 0;
        if (inb) {
            h = a.q[qid];
            const double hu = a.q[qid + N2], hv = a.q[qid + 2 * N2];
            const double iv = (h > a.c.PosPresTOL) ? 1.0 / h : 0.0;
            su[s] = hu * iv; sv[s] = hv * iv;
        }
        __syncthreads();
        if (inb) {
            const int rb = el * N2 + eta * NGL, cb = el * N2 + xi;
            const double J = a.Jinv[xid];
            const double ye = a.Yeta[xid], yx = a.Yxi[xid], xe = a.Xeta[xid], xx = a.Xxi[xid];
            double gx0, gx1, gy0, gy1;
            {
                double uxi = 0, ueta = 0, vxi = 0, veta = 0;
#pragma unroll
                for (int l = 0; l < NGL; ++l) {
                    uxi += sDh[xi * NGL + l] * su[rb + l];
                    ueta += sDh[eta * NGL + l] * su[cb + l * NGL];
                    vxi += sDh[xi * NGL + l] * sv[rb + l];
                    veta += sDh[eta * NGL + l] * sv[cb + l * NGL];
                }
                const double ux = ye * uxi - yx * ueta, vx = ye * vxi - yx * veta;
                const double uy = -xe * uxi + xx * ueta, vy = -xe * vxi + xx * veta;
                gx0 = J * ux; gx1 = J * vx; gy0 = J * uy; gy1 = J * vy;
            }
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                int side = -1, j = 0;
                if (pass == 0) {
                    if (eta == 0) { side = 0; j = xi; }
                    else if (eta == NGL - 1) { side = 2; j = xi; }
                } else {
                    if (xi == NGL - 1) { side = 1; j = eta; }
                    else if (xi == 0) { side = 3; j = eta; }
                }
                if (side >= 0) {
                    const int4 sd = a.side[(long)e * 4 + side];
                    const int inc = sd.z ? j : NGL - 1 - j;
                    const int ms = sd.y;
                    const double* ux = a.SGX + (long)sd.x * 2 * NGL + inc;
                    const double* uy = a.SGY + (long)sd.x * 2 * NGL + inc;
                    if (pass == 0) gx0 += ms * ux[0] * J;
                    else gx0 += ms * J * ux[0];
                    gx1 += ms * J * ux[NGL];
                    gy0 += ms * J * uy[0];
                    gy1 += ms * J * uy[NGL];
                }
            }
            const long gid = (long)e * 2 * N2 + nd;
            a.GX[gid] = h * gx0; a.GX[gid + N2] = h * gx1;
            a.GY[gid] = h * gy0; a.GY[gid + N2] = h * gy1;
        }
        __syncthreads();
    }
}

// Positivity limiter (okl/Positivity/PosPres.okl:17-223), optionally with the
// wave-speed maximum of the limited state.
template <int NGL>
__global__ void __launch_bounds__(ElemShape<NGL>::THREADS) k_pospres(int K, const double* __restrict__ EleSizes,
                                                                   const double* __restrict__ GLw,
                                                                   const double* __restrict__ Jinv, double* q,
                                                                   const int* __restrict__ elem_inst, DevState* st,
                                                                   int lam_flag, PhysConst c) {
    constexpr int N2 = NGL * NGL, NE = ElemShape<NGL>::NE;
    __shared__ double sH[NE * N2], sU[NE * N2], sVv[NE * N2], sJ[NE * N2];
    __shared__ double sAvg[NE][4];
    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    const int e0 = blockIdx.x * NE;
    const int e = e0 + el;
    const bool inb = e < K;
    const int ins = inb ? inst_of(elem_inst, e) : 0;
    const bool active = inb && !st[ins].done;
    const long qid = (long)e * 3 * N2 + nd;
    const int s = el * N2 + nd;
    if (active) {
        sH[s] = q[qid]; sU[s] = q[qid + N2]; sVv[s] = q[qid + 2 * N2];
        sJ[s] = Jinv[(long)e * N2 + nd];
    }
    __syncthreads();
    if (active && nd == 0) {
        double hmin = 0.0, ha = 0.0, hua = 0.0, hva = 0.0;
        for (int l = 0; l < NGL; ++l)
            for (int k = 0; k < NGL; ++k) {
                const int p = el * N2 + k * NGL + l;
                const double w = GLw[l] * GLw[k] / sJ[p];
                ha += sH[p] * w;
                hua += sU[p] * w;
                hva += sVv[p] * w;
                hmin = fmin(hmin, sH[p]);
            }
        const double es = EleSizes[e];
        ha = ha / es;
        if (fabs(ha) < c.ZeroTOL) ha = 0.0;
        sAvg[el][0] = ha;
        sAvg[el][1] = hua / es;
        sAvg[el][2] = hva / es;
        sAvg[el][3] = hmin;
    }
    __syncthreads();
    double lam = 0.0;
    if (active) {
        const double ha = sAvg[el][0], hua = sAvg[el][1], hva = sAvg[el][2], hmin = sAvg[el][3];
        const double theta = (ha == hmin) ? 1.0 : fmin(1.0, ha / (ha - hmin));
        double h = sH[s], hu = sU[s], hv = sVv[s];
        if (hmin < 0.0) {
            double hn = 0.0, hun = 0.0, hvn = 0.0;
            if (ha > 0.0) {
                hn = fabs(theta * (h - ha) + ha);
                if (hn > c.PosPresTOL) {
                    hun = theta * (hu - hua) + hua;
                    hvn = theta * (hv - hva) + hva;
                }
            }
            if (ha < 0.0) { hn = -1.0 / 0.0; hun = 0.0; hvn = 0.0; }  // -inf marks a failed limiter
            h = hn; hu = hun; hv = hvn;
            q[qid] = h; q[qid + N2] = hu; q[qid + 2 * N2] = hv;
        } else if (h < c.PosPresTOL) {
            hu = 0.0; hv = 0.0;
            q[qid + N2] = 0.0; q[qid + 2 * N2] = 0.0;
        }
        if (lam_flag) lam = node_lambda(c, h, hu, hv);
    }
    if (lam_flag) warp_lambda<ElemShape<NGL>::THREADS>(lam, active, ins, st);
}

// Wave-speed maximum of q (start of the time loop).
template <int NGL>
__global__ void __launch_bounds__(ElemShape<NGL>::THREADS) k_lambda(int K, const double* __restrict__ q,
                                                                  const int* __restrict__ elem_inst, DevState* st,
                                                                  PhysConst c) {
    constexpr int N2 = NGL * NGL, NE = ElemShape<NGL>::NE;
    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    const int e0 = blockIdx.x * NE;
    const int e = e0 + el;
    const bool inb = e < K;
    double lam = 0.0;
    const int ins = inb ? inst_of(elem_inst, e) : 0;
    if (inb) {
        const long qid = (long)e * 3 * N2 + nd;
        lam = node_lambda(c, q[qid], q[qid + N2], q[qid + 2 * N2]);
    }
    warp_lambda<ElemShape<NGL>::THREADS>(lam, inb, ins, st);
}

// Step bookkeeping per instance (src/deviceclass.cpp:897-930 and :1130):
// dt from the CFL and viscous limits, done flag when t >= T or the step cap
// is reached.
__global__ void k_step_begin(int I, DevState* st, int ngl, int AV) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= I) return;
    DevState& s = st[k];
    if (s.done) return;
    if (!(s.t < s.T) || (s.max_steps > 0 && s.steps >= s.max_steps)) { s.done = 1; return; }
    if (s.pause_on && s.steps > s.resume_steps && s.t >= s.pause_at) { s.done = 1; return; }
    const double lam = __longlong_as_double((long long)s.lam_key);
    if (s.lam_key == ~0ull || !isfinite(lam)) { s.status = ST_NONFINITE; s.done = 1; return; }
    const double dt_i = s.minEle / (double)ngl * s.CFL / lam;
    double dt;
    if (AV) {
        const double vmax = __longlong_as_double((long long)s.visc_key);
        const double dt_v = s.DFL / (pow((double)ngl, 2)) * pow(s.minEle, 2) / vmax;
        dt = fmin(s.T - s.t, fmin(dt_i, dt_v));
    } else {
        dt = fmin(s.T - s.t, dt_i);
    }
    s.dt = dt;
    s.lam_key = 0ull;
    s.visc_key = 0ull;
}

__global__ void k_step_end(int I, DevState* st) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= I) return;
    DevState& s = st[k];
    if (s.done) return;
    s.t += s.dt;
    s.steps += 1;
}

}  // namespace esdg
