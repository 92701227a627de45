// Element kernel with two nodes per thread: the same tiles, bulk-copy
// pipeline and per-node arithmetic as k_element_tma (every operation in the
// same order, so the same bits), with thread t working on node nd of
// element el and of element el + NE/2 of the tile.
//
// The two nodes share their position (xi, eta), hence their rows of the
// flux-differencing matrix, which stay in registers for the whole kernel
// instead of being read from shared memory per pair; and the two flux
// chains are independent, so the FP64 latency of one is covered by the
// other.  Half as many threads per tile as nodes: the per-thread overhead
// (tile loop, waits, index arithmetic) is paid once for two nodes.
#pragma once

#include "esdg_tma.cuh"

namespace esdg {

template <int NGL>
struct PairShape : TileLayout<NGL, TmaShape<NGL>::NE - TmaShape<NGL>::NE % 2> {
    using L = TileLayout<NGL, TmaShape<NGL>::NE - TmaShape<NGL>::NE % 2>;
    static_assert(L::NE >= 2, "two elements per tile at least");
    static constexpr int HALF = L::NE / 2;
    static constexpr int THREADS = HALF * L::N2;
    static constexpr int ST = 2;
    // shared layout: [ST][stage] | su, sv, sh2 [ND each] | mbar[ST]
    static constexpr size_t SMEM = sizeof(double) * (ST * (size_t)L::STAGE_DOUBLES + 3 * L::ND) + 16 * ST;
};

constexpr int PAIR_VARIANTS = 2;
__host__ __device__ constexpr int pair_min_blocks(int v) { return v == 0 ? 3 : 4; }

// GEN as for k_element_tma: 0 plain single mesh, 2 arena or active set
// without partial-dry treatment or manufactured source, 1 everything.
template <int NGL, int MINB, int GEN = 1>
__global__ void __launch_bounds__(PairShape<NGL>::THREADS, MINB) k_element_pair(ElemArgs a, int ntiles) {
    using P = PairShape<NGL>;
    constexpr int N2 = P::N2, NE = P::NE, H = P::HALF, ST = P::ST;
    if (GEN != 0 && a.extent) ntiles = min(ntiles, (a.extent[0] + NE - 1) / NE);
    extern __shared__ __align__(128) double smem[];
    double* stage = smem;
    double* su = smem + ST * P::STAGE_DOUBLES;
    double* sv = su + P::ND;
    double* sh2 = sv + P::ND;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sh2 + P::ND);
    const int tid = threadIdx.x;
    const int el0 = tid / N2, nd = tid % N2;  // nodes nd of elements el0 and el0 + H
    const int xi = nd % NGL, eta = nd / NGL;
    double Dx[NGL], De[NGL];  // rows xi and eta of the flux-differencing matrix
#pragma unroll
    for (int l = 0; l < NGL; ++l) {
        Dx[l] = a.D[xi * NGL + l];
        De[l] = a.D[eta * NGL + l];
    }
    if (tid == 0)
        for (int k = 0; k < ST; ++k) mbar_init(&bar[k], 1);
    __syncthreads();
    if (tid == 0)
        for (int k = 0; k < ST; ++k) {
            const int t = blockIdx.x + k * gridDim.x;
            if (t < ntiles) tile_issue<NGL, NE>(a, t, stage + k * P::STAGE_DOUBLES, &bar[k]);
        }
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int sidx = it % ST;
        const unsigned parity = (unsigned)((it / ST) & 1);
        double* sb = stage + sidx * P::STAGE_DOUBLES;
        const double* sq = sb;
        const double* s2 = sb + P::QD;
        const double* sJ = sb + 2 * P::QD;
        const double* sBx = sJ + P::ND;
        const double* sBy = sJ + 2 * P::ND;
        const double* sYx = sJ + 3 * P::ND;
        const double* sYe = sJ + 4 * P::ND;
        const double* sXx = sJ + 5 * P::ND;
        const double* sXe = sJ + 6 * P::ND;
        const double* sFt = sJ + 7 * P::ND;
        const int e0 = t * NE;
        int e[2], ins[2];
        bool active[2], to_list[2];
        double dt[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            e[k] = e0 + el0 + k * H;
            const bool inb = e[k] < a.K;
            ins[k] = (GEN != 0 && inb) ? inst_of(a.elem_inst, e[k]) : 0;
            active[k] = inb && !a.st[ins[k]].done;
            to_list[k] = GEN != 0 && active[k] && a.act && a.act[e[k]] != 0;
            dt[k] = (active[k] && a.mode != 2) ? a.st[ins[k]].dt : 0.0;
        }
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
        double h[2], hu[2], hv[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int s = (el0 + k * H) * N2 + nd, qs = (el0 + k * H) * 3 * N2 + nd;
            h[k] = sq[qs]; hu[k] = sq[qs + N2]; hv[k] = sq[qs + 2 * N2];
            const double ih = (h[k] > 0) ? 1.0 / h[k] : 0.0;
            su[s] = hu[k] * ih;
            sv[s] = hv[k] * ih;
            sh2[s] = h[k] * h[k];
        }
        __syncthreads();
        // flux-differencing sums of both nodes, interleaved pair by pair
        // (an inactive node's sums are computed and dropped)
        double d1[2] = {0.0, 0.0}, d2[2] = {0.0, 0.0}, d3[2] = {0.0, 0.0};
        const double g = a.c.g;
#pragma unroll
        for (int l = 0; l < NGL; ++l) {
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int s = (el0 + k * H) * N2 + nd;
                const int p = (el0 + k * H) * N2 + eta * NGL + l, pq = (el0 + k * H) * 3 * N2 + eta * NGL + l;
                double f1, f2, f3;
                pair_flux_raw<false>(g, h[k], hu[k], hv[k], su[s], sv[s], sh2[s], sYe[s], sXe[s], sq[pq],
                                     sq[pq + N2], sq[pq + 2 * N2], su[p], sv[p], sh2[p], sYe[p], sXe[p], f1, f2, f3);
                d1[k] += Dx[l] * f1; d2[k] += Dx[l] * f2; d3[k] += Dx[l] * f3;
            }
        }
#pragma unroll
        for (int l = 0; l < NGL; ++l) {
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int s = (el0 + k * H) * N2 + nd;
                const int p = (el0 + k * H) * N2 + xi + l * NGL, pq = (el0 + k * H) * 3 * N2 + xi + l * NGL;
                double g1, g2, g3;
                pair_flux_raw<true>(g, h[k], hu[k], hv[k], su[s], sv[s], sh2[s], sYx[s], sXx[s], sq[pq],
                                    sq[pq + N2], sq[pq + 2 * N2], su[p], sv[p], sh2[p], sYx[p], sXx[p], g1, g2, g3);
                d1[k] += De[l] * g1; d2[k] += De[l] * g2; d3[k] += De[l] * g3;
            }
        }
        double lam[2] = {0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (!active[k]) continue;
            const int el = el0 + k * H;
            const int s = el * N2 + nd, qs = el * 3 * N2 + nd;
            const double e1 = d1[k] * 0.25;
            const double e2 = d2[k] * 0.125;
            const double e3 = d3[k] * 0.125;
            const double J = sJ[s];
            double r0 = -J * e1;
            double r1 = -J * e2 - a.c.g * h[k] * sBx[s];
            double r2 = -J * e3 - a.c.g * h[k] * sBy[s];
            if (GEN == 1 && a.dry && a.dry[e[k]])
                pd_volume<NGL>(a.c, a.Dc, a.Dup, a.Ddn, sq + el * 3 * N2, a.Bn + (long)e[k] * N2, eta, xi, sYe[s],
                               sYx[s], sXe[s], sXx[s], J, r1, r2);
            // lift: sides 0/2 first, then 1/3, from the tile's element-side
            // fluxes (-ms * flux; DBSurf1/2 are zero)
            const double db = 0.0;
            const double* sF = sFt + el * 12 * NGL;
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
            if (GEN == 1 && a.conv) add_conv_source(a, a.st[ins[k]], (long)e[k] * N2 + nd, sBx[s], sBy[s], r0, r1, r2);
            const long qid = (long)e[k] * 3 * N2 + nd;
            if (a.mode == 2 || to_list[k]) {
                a.Qt[qid] = r0; a.Qt[qid + N2] = r1; a.Qt[qid + 2 * N2] = r2;
                if (to_list[k] && nd == 0) a.alist[atomicAdd(a.acount, 1)] = e[k];
            } else {
                const double o0 = s2[qs], o1 = s2[qs + N2], o2 = s2[qs + 2 * N2];
                double q0, q1, q2;
                if (a.mode == 0) {
                    const double g0 = a.rkA * o0 + r0;
                    const double g1 = a.rkA * o1 + r1;
                    const double g2 = a.rkA * o2 + r2;
                    a.gRK[qid] = g0; a.gRK[qid + N2] = g1; a.gRK[qid + 2 * N2] = g2;
                    q0 = h[k] + a.rkC * dt[k] * g0;
                    q1 = hu[k] + a.rkC * dt[k] * g1;
                    q2 = hv[k] + a.rkC * dt[k] * g2;
                } else {
                    q0 = a.rkA * o0 + a.rkB * h[k] + a.rkC * dt[k] * r0;
                    q1 = a.rkA * o1 + a.rkB * hu[k] + a.rkC * dt[k] * r1;
                    q2 = a.rkA * o2 + a.rkB * hv[k] + a.rkC * dt[k] * r2;
                }
                a.q[qid] = q0; a.q[qid + N2] = q1; a.q[qid + 2 * N2] = q2;
                if (a.lam) lam[k] = node_lambda(a.c, q0, q1, q2);
            }
        }
        if (a.lam) {
            warp_lambda<P::THREADS>(lam[0], active[0] && !to_list[0], ins[0], a.st);
            warp_lambda<P::THREADS>(lam[1], active[1] && !to_list[1], ins[1], a.st);
        }
        __syncthreads();  // stage buffer and su, sv, sh2 free again
        if (tid == 0) {
            const int tn = t + ST * gridDim.x;
            if (tn < ntiles) {
                fence_proxy_async_smem();
                tile_issue<NGL, NE>(a, tn, sb, &bar[sidx]);
            }
        }
    }
}

}  // namespace esdg
