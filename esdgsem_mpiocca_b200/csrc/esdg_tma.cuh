// Bulk-copy (TMA, cp.async.bulk) pipeline helpers for sm_100a and the
// persistent, double-buffered element kernel built on them.
//
// Each CTA walks tiles of NE consecutive elements (tile = blockIdx.x,
// blockIdx.x + gridDim.x, ...).  One thread issues, per tile, ten 1-D bulk
// copies global -> shared (q, gRK or Qtmp, Jinv, Bx, By, Y_xi, Y_eta, X_xi,
// X_eta and the element-side face fluxes: all contiguous in the
// element-major layout) completing on the stage's mbarrier; while the CTA
// computes tile k the copies of tile k+1 are in flight.  The arithmetic per
// node is that of k_element (same operands, same order), only the staging
// differs: no load of the compute phase leaves the shared memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "esdg_kernels.cuh"

namespace esdg {

enum : int { ST_TIMEOUT = 2 };

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// 1-D bulk copy global -> shared; dst, src and bytes are multiples of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Waits for the phase with the given parity; gives up after `limit` clock
// cycles (0: 4e9, about 2 s; a copy that never lands), returning false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, long long limit = 0) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long lim = limit > 0 ? limit : 4000000000ll;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > lim) return false;
    return true;
}

// After a wait ran out: the bulk copies of the stages still in flight
// (iterations it+1 .. it+ST-1 of this CTA) land before the CTA returns and
// its shared memory is released; bounded like every wait.  One thread.
template <int ST>
__device__ __forceinline__ void drain_stages(uint64_t* bar, int it, int t, int ntiles, int skip_tile,
                                             long long limit) {
#pragma unroll
    for (int k = 1; k < ST; ++k) {
        const int itk = it + k;
        const int tk = t + k * (int)gridDim.x;
        if (tk < ntiles && tk + 1 != skip_tile) mbar_wait_bounded(&bar[itk % ST], (unsigned)((itk / ST) & 1), limit);
    }
}

// Entropy-conservative two-point flux of okl/DG/VolumeKernelFluxDiffV99.okl:17-57,
// evaluated on raw sums.  Every average there is 0.5*(L+R) and every
// product of two averages then carries a factor 1/4 or 1/8; scaling by a
// power of two commutes exactly with IEEE rounding (no subnormals here), so
//   F1 = (Sa*Shu - Sb*Shv) / 4,
//   F2 = (Sa*(Shu*Su + P4) - (Sb*Shv)*Su) / 8,
//   F3 = (Sa*(Shu*Sv) - Sb*(Shv*Sv + P4)) / 8,   P4 = (g*Sh)*Sh - g*Sh2 = 4p,
// with S* = L+R (u = hu*(1/h), v, h2 = h*h formed once per node, as the
// reference forms them inside every pair), are the reference's values times
// 4 resp. 8, bit for bit.  The caller accumulates D*F on the unscaled values
// and applies 1/4 and 1/8 once per node, which is exact for the same reason.
// ETA selects G = -a f + b g instead of F = a f - b g.
template <bool ETA>
__device__ __forceinline__ void pair_flux_raw(double g, double hL, double huL, double hvL, double uL, double vL,
                                              double h2L, double aL, double bL, double hR, double huR, double hvR,
                                              double uR, double vR, double h2R, double aR, double bR, double& X1,
                                              double& X2, double& X3) {
    const double Sh = hL + hR;
    const double Sh2 = h2L + h2R;
    const double Shu = huL + huR;
    const double Shv = hvL + hvR;
    const double Su = uL + uR;
    const double Sv = vL + vR;
    const double Sa = aL + aR;
    const double Sb = bL + bR;
    const double P4 = g * Sh * Sh - g * Sh2;
    const double bhv = Sb * Shv;
    if (!ETA) {
        X1 = Sa * Shu - bhv;
        X2 = Sa * (Shu * Su + P4) - bhv * Su;
        X3 = Sa * (Shu * Sv) - Sb * (Shv * Sv + P4);
    } else {
        X1 = -Sa * Shu + bhv;
        X2 = -Sa * (Shu * Su + P4) + bhv * Su;
        X3 = -Sa * (Shu * Sv) + Sb * (Shv * Sv + P4);
    }
}

// Variants of the element kernel: CTAs per SM the register budget is cut
// for, and depth of the bulk-copy pipeline; the engine times them on the
// mesh and keeps the fastest.
constexpr int TMA_VARIANTS = 3;
__host__ __device__ constexpr int tma_min_blocks(int v) { return v == 1 ? 3 : 2; }
__host__ __device__ constexpr int tma_stages(int v) { return v == 2 ? 3 : 2; }

// One stage buffer of a tile of NE elements: q, gRK (or Qtmp), Jinv, Bx,
// By, Y_xi, Y_eta, X_xi, X_eta and the element-side face fluxes, each a
// contiguous section (NE * N2 even: every section starts on 16 bytes).
template <int NGL, int NE_>
struct TileLayout {
    static constexpr int N2 = NGL * NGL;
    static constexpr int NE = NE_;
    static_assert((NE * N2) % 2 == 0, "16-byte bulk granularity needs NE * N2 even");
    static constexpr int QD = NE * 3 * N2;    // doubles of a q-like section
    static constexpr int ND = NE * N2;        // doubles of a nodal section
    static constexpr int FD = NE * 12 * NGL;  // element-side face fluxes of the tile
    static constexpr int STAGE_DOUBLES = 2 * QD + 7 * ND + FD;
};

// elements per tile of the node-per-thread kernel: ~256 threads, NE*N2 even
__host__ __device__ constexpr int tma_ne(int n2) {
    return ((256 / n2) > 0 ? (256 / n2) : 1) % 2 == 1 && n2 % 2 == 1
               ? ((256 / n2) > 1 ? (256 / n2) - 1 : 2)
               : ((256 / n2) > 0 ? (256 / n2) : 1);
}

template <int NGL, int ST = 2>
struct TmaShape : TileLayout<NGL, tma_ne(NGL * NGL)> {
    using L = TileLayout<NGL, tma_ne(NGL * NGL)>;
    static constexpr int THREADS = L::NE * L::N2;
    static constexpr int STAGES = ST;
    // shared layout: [STAGES][stage] | su, sv, sh2 [ND each] | sD[N2] | mbar[STAGES]
    static constexpr size_t SMEM =
        sizeof(double) * (STAGES * (size_t)L::STAGE_DOUBLES + 3 * L::ND + L::N2) + 16 * STAGES;
};

// Issues the bulk copies of tile t (NE elements) into stage buffer sb (one
// thread).
template <int NGL, int NE>
__device__ __forceinline__ void tile_issue(const ElemArgs& a, int t, double* sb, uint64_t* bar) {
    using S = TileLayout<NGL, NE>;
    if (t + 1 == a.skip_tile) return;  // test hook: this tile's copies are never issued
    const int e0 = t * S::NE;
    const int ne = min(S::NE, a.K - e0);
    const unsigned qb = (unsigned)(ne * 3 * S::N2 * sizeof(double));
    const unsigned nb = (unsigned)(ne * S::N2 * sizeof(double));
    const unsigned fb = (unsigned)(ne * 12 * NGL * sizeof(double));
    const double* second = (a.mode == 1) ? a.Qtmp : a.gRK;
    const bool need2 = a.mode != 2;
    mbar_arrive_expect_tx(bar, qb + (need2 ? qb : 0u) + 7u * nb + fb);
    const long qo = (long)e0 * 3 * S::N2, no = (long)e0 * S::N2;
    bulk_g2s(sb + 2 * S::QD + 7 * S::ND, a.SP + side_flux_at(e0, 0, 0, 0, NGL), fb, bar);
    bulk_g2s(sb, a.q + qo, qb, bar);
    if (need2) bulk_g2s(sb + S::QD, second + qo, qb, bar);
    double* nd = sb + 2 * S::QD;
    bulk_g2s(nd + 0 * S::ND, a.Jinv + no, nb, bar);
    bulk_g2s(nd + 1 * S::ND, a.Bx + no, nb, bar);
    bulk_g2s(nd + 2 * S::ND, a.By + no, nb, bar);
    bulk_g2s(nd + 3 * S::ND, a.Yxi + no, nb, bar);
    bulk_g2s(nd + 4 * S::ND, a.Yeta + no, nb, bar);
    bulk_g2s(nd + 5 * S::ND, a.Xxi + no, nb, bar);
    bulk_g2s(nd + 6 * S::ND, a.Xeta + no, nb, bar);
}

template <int NGL>
__device__ __forceinline__ void tma_issue_tile(const ElemArgs& a, int t, double* sb, uint64_t* bar) {
    tile_issue<NGL, TmaShape<NGL>::NE>(a, t, sb, bar);
}

// Persistent flux-differencing volume term + surface lift + RK update
// (same operations as k_element), tiles double-buffered through TMA.
// GEN = 0: the plain single-mesh step (no arena, active set, partial-dry
// treatment or manufactured source), those branches compiled out; 2: an
// arena or active set without the partial-dry treatment and manufactured
// source; 1: everything.
template <int NGL, int MINB, int NST, int GEN = 1>
__global__ void __launch_bounds__(TmaShape<NGL>::THREADS, MINB) k_element_tma(ElemArgs a, int ntiles) {
    using S = TmaShape<NGL, NST>;
    constexpr int N2 = S::N2, NE = S::NE, ST = S::STAGES;
    if (GEN != 0 && a.extent) ntiles = min(ntiles, (a.extent[0] + NE - 1) / NE);
    extern __shared__ __align__(128) double smem[];
    double* stage = smem;
    double* su = smem + ST * S::STAGE_DOUBLES;
    double* sv = su + S::ND;
    double* sh2 = sv + S::ND;
    double* sD = sh2 + S::ND;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sD + N2);
    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    const int xi = nd % NGL, eta = nd / NGL;
    if (tid < N2) sD[tid] = a.D[tid];
    if (tid == 0)
        for (int k = 0; k < ST; ++k) mbar_init(&bar[k], 1);
    __syncthreads();
    if (tid == 0)
        for (int k = 0; k < ST; ++k) {
            const int t = blockIdx.x + k * gridDim.x;
            if (t < ntiles) tma_issue_tile<NGL>(a, t, stage + k * S::STAGE_DOUBLES, &bar[k]);
        }
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int sidx = it % ST;
        const unsigned parity = (unsigned)((it / ST) & 1);
        double* sb = stage + sidx * S::STAGE_DOUBLES;
        const double* sq = sb;
        const double* s2 = sb + S::QD;
        const double* sJ = sb + 2 * S::QD;
        const double* sBx = sJ + S::ND;
        const double* sBy = sJ + 2 * S::ND;
        const double* sYx = sJ + 3 * S::ND;
        const double* sYe = sJ + 4 * S::ND;
        const double* sXx = sJ + 5 * S::ND;
        const double* sXe = sJ + 6 * S::ND;
        const int e0 = t * NE;
        const int e = e0 + el;
        const bool inb = e < a.K;
        const int ins = (GEN != 0 && inb) ? inst_of(a.elem_inst, e) : 0;
        const bool active = inb && !a.st[ins].done;
        const bool to_list = GEN != 0 && active && a.act && a.act[e] != 0;
        const double dt = (active && a.mode != 2) ? a.st[ins].dt : 0.0;
        // every thread waits for the tile; a copy that never lands makes the
        // whole CTA leave together (uniform decision) with an error status
        // for the host instead of hanging
        const bool landed = mbar_wait_bounded(&bar[sidx], parity, a.wait_limit);
        if (__syncthreads_or(!landed)) {
            if (tid == 0) {
                atomicExch(&a.st[0].status, ST_TIMEOUT);
                drain_stages<ST>(bar, it, t, ntiles, a.skip_tile, a.wait_limit);
            }
            return;
        }
        const int s = el * N2 + nd;          // node slot in nodal sections
        const int qs = el * 3 * N2 + nd;     // node slot in q sections
        double h = 0, hu = 0, hv = 0;
        if (active) {
            h = sq[qs]; hu = sq[qs + N2]; hv = sq[qs + 2 * N2];
            const double ih = (h > 0) ? 1.0 / h : 0.0;
            su[s] = hu * ih;
            sv[s] = hv * ih;
            sh2[s] = h * h;
        }
        __syncthreads();
        double lam = 0.0;
        if (active) {
            const int rb = el * N2 + eta * NGL, cb = el * N2 + xi;
            const int qrb = el * 3 * N2 + eta * NGL, qcb = el * 3 * N2 + xi;
            const double ye = sYe[s], yx = sYx[s], xe = sXe[s], xx = sXx[s];
            const double uL = su[s], vL = sv[s], h2L = sh2[s];
            const double g = a.c.g;
            double d1 = 0.0, d2 = 0.0, d3 = 0.0;
#pragma unroll
            for (int l = 0; l < NGL; ++l) {
                const int p = rb + l, pq = qrb + l;
                const double dl = sD[xi * NGL + l];
                double f1, f2, f3;
                pair_flux_raw<false>(g, h, hu, hv, uL, vL, h2L, ye, xe, sq[pq], sq[pq + N2], sq[pq + 2 * N2], su[p],
                                     sv[p], sh2[p], sYe[p], sXe[p], f1, f2, f3);
                d1 += dl * f1; d2 += dl * f2; d3 += dl * f3;
            }
#pragma unroll
            for (int l = 0; l < NGL; ++l) {
                const int p = cb + l * NGL, pq = qcb + l * NGL;
                const double dl = sD[eta * NGL + l];
                double g1, g2, g3;
                pair_flux_raw<true>(g, h, hu, hv, uL, vL, h2L, yx, xx, sq[pq], sq[pq + N2], sq[pq + 2 * N2], su[p],
                                    sv[p], sh2[p], sYx[p], sXx[p], g1, g2, g3);
                d1 += dl * g1; d2 += dl * g2; d3 += dl * g3;
            }
            d1 *= 0.25;
            d2 *= 0.125;
            d3 *= 0.125;
            const double J = sJ[s];
            double r0 = -J * d1;
            double r1 = -J * d2 - a.c.g * h * sBx[s];
            double r2 = -J * d3 - a.c.g * h * sBy[s];
            if (GEN == 1 && a.dry && a.dry[e])
                pd_volume<NGL>(a.c, a.Dc, a.Dup, a.Ddn, sq + el * 3 * N2, a.Bn + (long)e * N2, eta, xi, ye, yx, xe, xx,
                               J, r1, r2);
            // lift: sides 0/2 first, then 1/3, from the tile's element-side
            // fluxes (-ms * flux; DBSurf1/2 are zero)
            const double db = 0.0;
            const double* sF = sJ + 7 * S::ND + el * 12 * NGL;
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
                    const double* fp = sF + side * 3 * NGL + j;
                    r0 += fp[0] * J;
                    r1 += J * fp[NGL] + J * db;
                    r2 += J * fp[2 * NGL] + J * db;
                }
            }
            if (GEN == 1 && a.conv) add_conv_source(a, a.st[ins], (long)e * N2 + nd, sBx[s], sBy[s], r0, r1, r2);
            const long qid = (long)e * 3 * N2 + nd;
            if (a.mode == 2 || to_list) {
                a.Qt[qid] = r0; a.Qt[qid + N2] = r1; a.Qt[qid + 2 * N2] = r2;
                if (to_list && nd == 0) a.alist[atomicAdd(a.acount, 1)] = e;
            } else {
                const double o0 = s2[qs], o1 = s2[qs + N2], o2 = s2[qs + 2 * N2];
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
        if (a.lam) warp_lambda<S::THREADS>(lam, active && !to_list, ins, a.st);
        __syncthreads();  // stage buffer and si free again
        if (tid == 0) {
            const int tn = t + ST * gridDim.x;
            if (tn < ntiles) {
                fence_proxy_async_smem();
                tma_issue_tile<NGL>(a, tn, sb, &bar[sidx]);
            }
        }
    }
}

}  // namespace esdg
