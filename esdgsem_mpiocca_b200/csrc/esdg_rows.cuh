// Line-per-thread element kernel: the same flux-differencing volume term,
// surface lift and RK update as k_element_tma, with one thread per element
// row (xi sums) and then per element column (eta sums) instead of one thread
// per node.
//
// The entropy-conservative two-point flux of okl/DG/VolumeKernelFluxDiffV99.okl:17-57
// depends on its two states only through sums (h_i + h_j, ...), so in IEEE
// arithmetic F(i,j) and F(j,i) are the same bits.  A thread that holds a
// whole line of NGL nodes in registers evaluates each of the NGL(NGL+1)/2
// pairs once and adds it to both nodes.  Visiting the pairs (i, l), i <= l,
// row by row gives every node its terms in partner order l = 0..NGL-1 --
// the order of the reference's loops (okl/DG/VolumeKernelFluxDiffV99.okl:166-200),
// so each node's sum rounds exactly as there.  The xi sums pass through
// shared memory to the column threads, which continue each node's sum with
// its eta terms, again in partner order.
//
// Per tile of NE elements one thread issues ten 1-D bulk copies (q, gRK or
// Qtmp, Jinv, Bx, By, Y_xi, Y_eta, X_xi, X_eta, the element-side face
// fluxes) into the
// stage's buffer; the updated q (and gRK) are written back into the same
// buffer and leave with one bulk store per array when every element of the
// tile is active and none is partly dry, by plain stores otherwise.  Thread
// t works on element t % NE, line t / NE: consecutive threads touch
// consecutive elements, whose shared-memory slots lie an odd number of
// doubles apart (3 N2 or N2 with N2 odd, or a multiple of 16 bytes apart
// with an odd quotient), so the accesses of a half-warp fall in distinct
// banks.
#pragma once

#include "esdg_tma.cuh"

namespace esdg {

// D of the flux-differencing sums as a kernel parameter: the arithmetic
// reads its entries as constant-bank operands, without load instructions.
template <int NGL>
struct DLine {
    double v[NGL * NGL];
};

template <int NGL, int NE_, int ST_>
struct RowShape {
    static constexpr int N2 = NGL * NGL;
    static constexpr int NE = NE_;
    static constexpr int ST = ST_;
    static_assert((NE * N2) % 2 == 0, "16-byte bulk granularity needs NE * N2 even");
    static constexpr int LINES = NE * NGL;  // working threads
    static constexpr int THREADS = (LINES + 31) / 32 * 32;
    static constexpr int QD = 3 * NE * N2;
    static constexpr int ND = NE * N2;
    static constexpr int FD = NE * 12 * NGL;  // element-side face fluxes of the tile
    static constexpr int STAGE_DOUBLES = 2 * QD + 7 * ND + FD;
    // shared layout: [ST][stage] | xi sums [3][ND] | mbar[ST]
    static constexpr size_t SMEM = sizeof(double) * ((size_t)ST * STAGE_DOUBLES + 3 * (size_t)ND) + 16 * ST;
};

// Elements per tile of the row kernel's variants: the largest of 32 (64
// for NGL = 2) that keeps two stages within 200 KB, and half of it.
__host__ __device__ constexpr size_t row_smem_bytes(int ngl, int ne, int st) {
    return sizeof(double) * ((size_t)st * (size_t)ne * (13 * ngl * ngl + 12 * ngl) + 3 * (size_t)ne * ngl * ngl) +
           16 * st;
}
__host__ __device__ constexpr int row_ne_fit(int ngl, int ne) {
    return (ne <= 2 || row_smem_bytes(ngl, ne, 2) <= 200 * 1024) ? ne : row_ne_fit(ngl, ne - 2);
}
constexpr int ROW_VARIANTS = 2;
__host__ __device__ constexpr int row_ne(int ngl, int r) {
    return r == 0 ? row_ne_fit(ngl, ngl == 2 ? 64 : 32) : (row_ne_fit(ngl, ngl == 2 ? 64 : 32) / 4) * 2;
}
__host__ __device__ constexpr int row_min_blocks(int r) { return r == 0 ? 1 : 2; }
// degrees the row kernel is compiled for
__host__ __device__ constexpr bool row_ngl_ok(int ngl) { return ngl >= 3 && ngl <= 6; }

__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the bulk stores issued by this thread have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// the bulk stores issued by this thread are complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Issues the bulk copies of tile t into stage buffer sb (one thread).
template <int NGL, int NE, int ST>
__device__ __forceinline__ void rows_issue_tile(const ElemArgs& a, int t, double* sb, uint64_t* bar) {
    using S = RowShape<NGL, NE, ST>;
    if (t + 1 == a.skip_tile) return;  // test hook: this tile's copies are never issued
    const int e0 = t * NE;
    const int ne = min(NE, a.K - e0);
    const unsigned qb = (unsigned)(ne * 3 * S::N2 * sizeof(double));
    const unsigned nb = (unsigned)(ne * S::N2 * sizeof(double));
    const unsigned fbytes = (unsigned)(ne * 12 * NGL * sizeof(double));
    const double* second = (a.mode == 1) ? a.Qtmp : a.gRK;
    const bool need2 = a.mode != 2;
    mbar_arrive_expect_tx(bar, qb + (need2 ? qb : 0u) + 7u * nb + fbytes);
    const long qo = (long)e0 * 3 * S::N2, no = (long)e0 * S::N2;
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
    bulk_g2s(nd + 7 * S::ND, a.SP + side_flux_at(e0, 0, 0, 0, NGL), fbytes, bar);
}

// Flux-differencing sums along one line of NGL nodes held in registers
// (ETA = false: a row, metric terms Y_eta, X_eta; ETA = true: a column,
// Y_xi, X_xi), each pair evaluated once, each node's terms added in partner
// order onto d1..d3.
template <int NGL, bool ETA>
__device__ __forceinline__ void line_sums(double g, const DLine<NGL>& Dm, const double (&h)[NGL],
                                          const double (&hu)[NGL], const double (&hv)[NGL], const double (&u)[NGL],
                                          const double (&v)[NGL], const double (&h2)[NGL], const double (&ma)[NGL],
                                          const double (&mb)[NGL], double (&d1)[NGL], double (&d2)[NGL],
                                          double (&d3)[NGL]) {
#pragma unroll
    for (int i = 0; i < NGL; ++i) {
#pragma unroll
        for (int l = i; l < NGL; ++l) {
            double f1, f2, f3;
            pair_flux_raw<ETA>(g, h[i], hu[i], hv[i], u[i], v[i], h2[i], ma[i], mb[i], h[l], hu[l], hv[l], u[l], v[l],
                               h2[l], ma[l], mb[l], f1, f2, f3);
            const double di = Dm.v[i * NGL + l];
            d1[i] += di * f1;
            d2[i] += di * f2;
            d3[i] += di * f3;
            if (l != i) {
                const double dl = Dm.v[l * NGL + i];
                d1[l] += dl * f1;
                d2[l] += dl * f2;
                d3[l] += dl * f3;
            }
        }
    }
}

// Loads the line's states and metric terms; u, v, h^2 formed per node as in
// k_element_tma.  Node j of the line sits at q slot qb + j * stride and
// nodal slot nb + j * stride.
template <int NGL>
__device__ __forceinline__ void line_load(const double* sq, const double* sa, const double* sbm, int qb, int nb,
                                          int stride, double (&h)[NGL], double (&hu)[NGL], double (&hv)[NGL],
                                          double (&u)[NGL], double (&v)[NGL], double (&h2)[NGL], double (&ma)[NGL],
                                          double (&mb)[NGL]) {
    constexpr int N2 = NGL * NGL;
#pragma unroll
    for (int j = 0; j < NGL; ++j) {
        const int qs = qb + j * stride, s = nb + j * stride;
        h[j] = sq[qs];
        hu[j] = sq[qs + N2];
        hv[j] = sq[qs + 2 * N2];
        const double ih = (h[j] > 0) ? 1.0 / h[j] : 0.0;
        u[j] = hu[j] * ih;
        v[j] = hv[j] * ih;
        h2[j] = h[j] * h[j];
        ma[j] = sa[s];
        mb[j] = sbm[s];
    }
}

// Persistent flux-differencing volume term + surface lift + RK update,
// one thread per element line, tiles double-buffered through bulk copies.
template <int NGL, int NE, int ST, int MINB>
__global__ void __launch_bounds__(RowShape<NGL, NE, ST>::THREADS, MINB)
    k_element_rows(ElemArgs a, DLine<NGL> Dm, int ntiles) {
    using S = RowShape<NGL, NE, ST>;
    constexpr int N2 = S::N2, ND = S::ND, QD = S::QD;
    if (a.extent) ntiles = min(ntiles, (a.extent[0] + NE - 1) / NE);
    extern __shared__ __align__(128) double smem[];
    double* stage = smem;
    double* sdx = smem + ST * S::STAGE_DOUBLES;  // xi sums [3][ND]
    uint64_t* bar = reinterpret_cast<uint64_t*>(sdx + 3 * ND);
    const int tid = threadIdx.x;
    const bool worker = tid < S::LINES;
    const int ln = worker ? tid / NE : 0;  // row (xi sums), then column (eta sums)
    const int el = worker ? tid % NE : 0;
    if (tid == 0)
        for (int k = 0; k < ST; ++k) mbar_init(&bar[k], 1);
    __syncthreads();
    if (tid == 0)
        for (int k = 0; k < ST; ++k) {
            const int t = blockIdx.x + k * gridDim.x;
            if (t < ntiles) rows_issue_tile<NGL, NE, ST>(a, t, stage + k * S::STAGE_DOUBLES, &bar[k]);
        }
    const double g = a.c.g;
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int sidx = it % ST;
        const unsigned parity = (unsigned)((it / ST) & 1);
        double* sb = stage + sidx * S::STAGE_DOUBLES;
        double* sq = sb;
        double* s2 = sb + QD;
        const double* sJ = sb + 2 * QD;
        const double* sBx = sJ + ND;
        const double* sBy = sJ + 2 * ND;
        const double* sYx = sJ + 3 * ND;
        const double* sYe = sJ + 4 * ND;
        const double* sXx = sJ + 5 * ND;
        const double* sXe = sJ + 6 * ND;
        const double* sF = sJ + 7 * ND;  // element-side face fluxes [NE][4][3][NGL]
        const int e0 = t * NE;
        const int e = e0 + el;
        const bool inb = worker && e < a.K;
        const int ins = inb ? inst_of(a.elem_inst, e) : 0;
        const bool active = inb && !a.st[ins].done;
        const bool to_list = active && a.act && a.act[e] != 0;
        const double dt = (active && a.mode != 2) ? a.st[ins].dt : 0.0;
        // a copy that never lands makes the whole CTA leave together
        // (uniform decision) with an error status for the host
        const bool landed = mbar_wait_bounded(&bar[sidx], parity, a.wait_limit);
        if (__syncthreads_or(!landed)) {
            if (tid == 0) {
                atomicExch(&a.st[0].status, ST_TIMEOUT);
                drain_stages<ST>(bar, it, t, ntiles, a.skip_tile, a.wait_limit);
                bulk_wait_all();
            }
            return;
        }
        // ---- xi sums: row ln of element el ----
        if (active) {
            double h[NGL], hu[NGL], hv[NGL], u[NGL], v[NGL], h2[NGL], ya[NGL], xa[NGL];
            const int qr = el * 3 * N2 + ln * NGL, nr = el * N2 + ln * NGL;
            line_load<NGL>(sq, sYe, sXe, qr, nr, 1, h, hu, hv, u, v, h2, ya, xa);
            double d1[NGL], d2[NGL], d3[NGL];
#pragma unroll
            for (int j = 0; j < NGL; ++j) d1[j] = d2[j] = d3[j] = 0.0;
            line_sums<NGL, false>(g, Dm, h, hu, hv, u, v, h2, ya, xa, d1, d2, d3);
#pragma unroll
            for (int j = 0; j < NGL; ++j) {
                sdx[nr + j] = d1[j];
                sdx[ND + nr + j] = d2[j];
                sdx[2 * ND + nr + j] = d3[j];
            }
        }
        // every element of the tile active: the update goes back through the
        // stage buffer and one bulk store per array
        // also the barrier between the two sums; a partly dry element reads
        // its neighbours' old h in the update, so such tiles store directly
        const int idle = __syncthreads_or((inb && !active) || (active && a.dry && a.dry[e]));
        const bool bulk = (a.mode != 2) && !idle;
        // ---- eta sums, surface lift and update: column ln of element el ----
        double lam = 0.0;
        if (active) {
            const int qc = el * 3 * N2 + ln, nc = el * N2 + ln;
            // the column's boundary nodes take the element-side fluxes
            // (-ms * flux) of sides 0 (j = 0) and 2 (j = NGL-1) in eta, 1
            // (ln = NGL-1) or 3 (ln = 0) in xi
            const double* fel = sF + el * 12 * NGL;
            const bool xedge = (ln == 0) || (ln == NGL - 1);
            const double* fx = fel + (ln == NGL - 1 ? 1 : 3) * 3 * NGL;
            double h[NGL], hu[NGL], hv[NGL], u[NGL], v[NGL], h2[NGL], yx[NGL], xx[NGL];
            line_load<NGL>(sq, sYx, sXx, qc, nc, NGL, h, hu, hv, u, v, h2, yx, xx);
            double d1[NGL], d2[NGL], d3[NGL];
#pragma unroll
            for (int j = 0; j < NGL; ++j) {
                const int s = nc + j * NGL;
                d1[j] = sdx[s];
                d2[j] = sdx[ND + s];
                d3[j] = sdx[2 * ND + s];
            }
            line_sums<NGL, true>(g, Dm, h, hu, hv, u, v, h2, yx, xx, d1, d2, d3);
            const long qe = (long)e * 3 * N2 + ln;
#pragma unroll
            for (int j = 0; j < NGL; ++j) {
                const int s = nc + j * NGL, qs = qc + j * NGL;
                const double e1 = d1[j] * 0.25;
                const double e2 = d2[j] * 0.125;
                const double e3 = d3[j] * 0.125;
                const double J = sJ[s];
                double r0 = -J * e1;
                double r1 = -J * e2 - a.c.g * h[j] * sBx[s];
                double r2 = -J * e3 - a.c.g * h[j] * sBy[s];
                if (a.dry && a.dry[e])
                    pd_volume<NGL>(a.c, a.Dc, a.Dup, a.Ddn, sq + el * 3 * N2, a.Bn + (long)e * N2, j, ln, sYe[s],
                                   sYx[s], sXe[s], sXx[s], J, r1, r2);
                const double db = 0.0;
                if (j == 0 || j == NGL - 1) {  // eta sides (0 at j = 0, 2 at j = NGL-1), node ln along them
                    const double* f = fel + (j == 0 ? 0 : 2) * 3 * NGL + ln;
                    r0 += f[0] * J;
                    r1 += J * f[NGL] + J * db;
                    r2 += J * f[2 * NGL] + J * db;
                }
                if (xedge) {  // xi side (1 at ln = NGL-1, 3 at ln = 0), node j along it
                    r0 += fx[j] * J;
                    r1 += J * fx[NGL + j] + J * db;
                    r2 += J * fx[2 * NGL + j] + J * db;
                }
                if (a.conv) add_conv_source(a, a.st[ins], (long)e * N2 + j * NGL + ln, sBx[s], sBy[s], r0, r1, r2);
                const long qid = qe + j * NGL;
                if (a.mode == 2 || to_list) {
                    a.Qt[qid] = r0; a.Qt[qid + N2] = r1; a.Qt[qid + 2 * N2] = r2;
                } else {
                    const double o0 = s2[qs], o1 = s2[qs + N2], o2 = s2[qs + 2 * N2];
                    double q0, q1, q2;
                    if (a.mode == 0) {
                        const double g0 = a.rkA * o0 + r0;
                        const double g1 = a.rkA * o1 + r1;
                        const double g2 = a.rkA * o2 + r2;
                        if (bulk) {
                            s2[qs] = g0; s2[qs + N2] = g1; s2[qs + 2 * N2] = g2;
                        } else {
                            a.gRK[qid] = g0; a.gRK[qid + N2] = g1; a.gRK[qid + 2 * N2] = g2;
                        }
                        q0 = h[j] + a.rkC * dt * g0;
                        q1 = hu[j] + a.rkC * dt * g1;
                        q2 = hv[j] + a.rkC * dt * g2;
                    } else {
                        q0 = a.rkA * o0 + a.rkB * h[j] + a.rkC * dt * r0;
                        q1 = a.rkA * o1 + a.rkB * hu[j] + a.rkC * dt * r1;
                        q2 = a.rkA * o2 + a.rkB * hv[j] + a.rkC * dt * r2;
                    }
                    if (bulk) {
                        sq[qs] = q0; sq[qs + N2] = q1; sq[qs + 2 * N2] = q2;
                    } else {
                        a.q[qid] = q0; a.q[qid + N2] = q1; a.q[qid + 2 * N2] = q2;
                    }
                    if (a.lam) {
                        const double lj = node_lambda(a.c, q0, q1, q2);
                        lam = (isnan(lj) || lj > lam) ? lj : lam;
                    }
                }
            }
            if (to_list && ln == 0) a.alist[atomicAdd(a.acount, 1)] = e;
        }
        if (a.lam) warp_lambda<S::THREADS>(lam, active && !to_list, ins, a.st);
        if (bulk) fence_proxy_async_smem();  // shared-memory writes before the bulk store reads them
        __syncthreads();                     // stage buffer and xi sums free again
        if (tid == 0) {
            if (bulk) {
                const int ne = min(NE, a.K - e0);
                const long qo = (long)e0 * 3 * N2;
                const unsigned qb = (unsigned)(ne * 3 * N2 * sizeof(double));
                bulk_s2g(a.q + qo, sq, qb);
                if (a.mode == 0) bulk_s2g(a.gRK + qo, s2, qb);
                bulk_commit();
            }
            const int tn = t + ST * gridDim.x;
            if (tn < ntiles) {
                if (bulk) bulk_wait_read_all();
                fence_proxy_async_smem();
                rows_issue_tile<NGL, NE, ST>(a, tn, sb, &bar[sidx]);
            }
        }
    }
    if (tid == 0) bulk_wait_all();
}

}  // namespace esdg
