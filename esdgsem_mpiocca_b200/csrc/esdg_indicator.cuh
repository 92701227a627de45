// Troubled-cell indicator with active-set marking (no counterpart in the
// reference, which evaluates the modal sensor and the whole viscous path
// on every element).
//
// Per element e it writes the artificial viscosity VP[e] and, where
// VP[e] > 0 and an active set is kept (act non-null), flags e and its face
// neighbours in act[] (zeroed before the launch).  Without act it is the
// reference path's sensor pass.  The viscous terms of an element vanish exactly unless it or a
// neighbour has VP > 0 (the face viscosity is max(VP_L, VP_R), the volume
// term is VP_e times the gradient), so the stage's viscous kernels run on
// the flagged elements only and give the same numbers as on all of them.
//
// LEARNED = false: the modal sensor (the arithmetic of
// okl/ShockCapturing/ShockCapturing.okl:17-234) on every element.
// LEARNED = true: the MLP (esdg_mlp.cuh) predicts sigma; its answer is
// used only where it is confident -- sigma_hat < sigma_min - margin gives
// VP = 0, sigma_hat > sigma_max + margin gives VP = eps0 -- and the modal
// sensor decides every other element: the ramp band, elements failing the
// positivity check (min h <= PosPresTOL or a non-finite value), and
// elements whose modal energy may be near the sensor's absolute ZeroTOL
// threshold (bounded from the nodal energy by emin/emax).
//
// Layout: like the element kernels, NE elements per block and one thread
// per node.  The modal transform runs one entry per thread (the same
// arithmetic as the serial loops), the order-dependent sums one thread per
// element.  For the network, one warp runs the block's (<= 16) feature rows
// through the tensor cores.
#pragma once

#include "esdg_mlp.cuh"

namespace esdg {

struct IndArgs {
    int K;
    const double* __restrict__ q;
    const double* __restrict__ B;
    const double* __restrict__ Vinv;
    double* __restrict__ VP;
    int* act;
    const int4* __restrict__ nbr;  // face neighbours (k_build_nbr)
    const int* __restrict__ extent = nullptr;  // live extent ([0] elements), as in FaceArgs
    const int* __restrict__ elem_inst;
    DevState* st;
    PhysConst c;
    int stage0;  // 1: fold VP into the instance's visc_key (dt of the step)
    // learned
    const float* __restrict__ P;
    const __nv_bfloat16* __restrict__ Pb;
    MlpLayout L;
    float margin;
    double emin, emax;  // n1 / sum(m^2) bounds of the modal energy
    // counts (optional): [0] zero by the net, [1] eps0 by the net,
    // [2] modal sensor, [3] elements with VP > 0
    unsigned long long* stats;
    // learned: the network's inputs and outputs per element (k_ind_features
    // and k_mlp_forward run first): feature rows X, s_eta, the nodal energy
    // sum(eta^2), the positivity/finiteness check, the network output y
    __nv_bfloat16* X;
    float* seta;
    double* energy;
    unsigned char* ok;
    float* y;
};

// Face neighbours of elements e0 .. e0+n-1 (-1 across walls): nbr[e] =
// the element on the other side of sides 0..3.
__global__ void k_build_nbr(int e0, int n, const int4* __restrict__ side, const int4* __restrict__ ftab,
                            int4* __restrict__ nbr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int e = e0 + i;
    int nb[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int4 t = ftab[side[(long)e * 4 + k].x];
        nb[k] = (t.x == e) ? t.y : t.x;
    }
    nbr[e] = make_int4(nb[0], nb[1], nb[2], nb[3]);
}

// Flags e and its face neighbours.
__device__ __forceinline__ void mark_active(int* act, int e, int4 nb) {
    act[e] = 1;
    if (nb.x >= 0) act[nb.x] = 1;
    if (nb.y >= 0) act[nb.y] = 1;
    if (nb.z >= 0) act[nb.z] = 1;
    if (nb.w >= 0) act[nb.w] = 1;
}

template <int NGL>
struct IndShape {
    static constexpr int N2 = NGL * NGL, NE = ElemShape<NGL>::NE, THREADS = NE * N2;
};


// Learned pass 1: feature rows and the decision inputs of every live
// element, for degrees whose element is an aligned group of lanes (n^2
// divides 32): NE elements per tile, one thread per node, the per-element
// sums by shuffles within the group, no block-wide barrier.  Persistent,
// the next tile's loads in flight while a tile is processed.
template <int NGL>
__global__ void __launch_bounds__(IndShape<NGL>::THREADS) k_ind_features(IndArgs a, int ntiles) {
    using S = IndShape<NGL>;
    constexpr int N2 = S::N2, NE = S::NE, KP = mlp_kp(NGL);
    static_assert((32 % N2) == 0, "element = aligned lane group");
    if (a.extent) ntiles = min(ntiles, (a.extent[0] + NE - 1) / NE);
    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    struct Ld {
        double h, b, hu, hv;
        int ins;
    };
    auto fetch = [&](int t) {
        Ld L{1.0, 0.0, 0.0, 0.0, -1};
        const int e = t * NE + el;
        if (e < a.K) {
            const long qid = (long)e * 3 * N2 + nd;
            L.h = a.q[qid];
            L.b = a.B[(long)e * N2 + nd];
            L.hu = a.q[qid + N2];
            L.hv = a.q[qid + 2 * N2];
            L.ins = inst_of(a.elem_inst, e);
        }
        return L;
    };
    int t = blockIdx.x;
    Ld nxt = (t < ntiles) ? fetch(t) : Ld{1.0, 0.0, 0.0, 0.0, -1};
    for (; t < ntiles; t += gridDim.x) {
        const Ld cur = nxt;
        if (t + gridDim.x < ntiles) nxt = fetch(t + gridDim.x);
        const int e = t * NE + el;
        const bool live = e < a.K && !a.st[cur.ins].done;
        const double v3[3] = {cur.b + cur.h, cur.hu, cur.hv};
        double mh = cur.h, e2 = v3[0] * v3[0];
        bool fin = isfinite(cur.h) && isfinite(cur.hu) && isfinite(cur.hv);
        double m3[3] = {v3[0], v3[1], v3[2]};
#pragma unroll
        for (int off = N2 / 2; off > 0; off >>= 1) {
#pragma unroll
            for (int f = 0; f < 3; ++f) m3[f] += __shfl_xor_sync(0xffffffffu, m3[f], off);
            mh = fmin(mh, __shfl_xor_sync(0xffffffffu, mh, off));
            e2 += __shfl_xor_sync(0xffffffffu, e2, off);
            fin = __shfl_xor_sync(0xffffffffu, (int)fin, off) && fin;
        }
        // deviations from the (double) mean; their statistics in single
        // precision, which is all the BF16 features need
        float dv[3], d3f[3];
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            m3[f] /= N2;
            dv[f] = (float)(v3[f] - m3[f]);
            d3f[f] = dv[f] * dv[f];
        }
#pragma unroll
        for (int off = N2 / 2; off > 0; off >>= 1)
#pragma unroll
            for (int f = 0; f < 3; ++f) d3f[f] += __shfl_xor_sync(0xffffffffu, d3f[f], off);
        if (!live) continue;  // after the shuffles: the whole group skips together
        __nv_bfloat16* xr = a.X + (long)e * KP;
        float rmsf[3];
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            rmsf[f] = sqrtf(d3f[f] * (1.0f / N2));
            const float mf = fabsf((float)m3[f]);
            const float inv = (rmsf[f] > (float)MLP_REL_FLAT * mf && rmsf[f] > 0.0f) ? 1.0f / rmsf[f] : 0.0f;
            xr[f * N2 + nd] = __float2bfloat16(dv[f] * inv);
        }
        if (nd < 3) {  // lanes 0, 1, 2 of the group: the scale feature of their field, one log10 pass
            const float r = nd == 0 ? rmsf[0] : (nd == 1 ? rmsf[1] : rmsf[2]);
            const float m = (float)(nd == 0 ? m3[0] : (nd == 1 ? m3[1] : m3[2]));
            const float tot = m * m + r * r;
            const float sf = (tot > 0.0f && r > 0.0f) ? fmaxf(log10f(r * r / tot), (float)MLP_S_MIN) : (float)MLP_S_MIN;
            xr[3 * N2 + nd] = __float2bfloat16(0.25f * sf);
            if (nd == 0) a.seta[e] = sf;
        }
        for (int c = 3 * N2 + 3 + nd; c < KP; c += N2) xr[c] = __float2bfloat16(0.0f);
        if (nd == 0) {
            a.energy[e] = e2;
            a.ok[e] = (fin && mh > a.c.PosPresTOL) ? 1 : 0;
        }
    }
}

// Learned pass 1 for degrees whose element is not an aligned lane group
// (n^2 does not divide 32): one warp per element (nodes lane, lane + 32,
// ...), the three fields' sums interleaved, no block-wide barrier.
template <int NGL>
__device__ __forceinline__ void ind_features_warp_elem(const IndArgs& a, int e) {
    constexpr int N2 = NGL * NGL, R = (N2 + 31) / 32, KP = mlp_kp(NGL);
    const int lane = threadIdx.x & 31;
    if (a.st[inst_of(a.elem_inst, e)].done) return;
    const double* qe = a.q + (long)e * 3 * N2;
    double v[3][R];
    double mh = 1e300, e2 = 0.0, m3[3] = {0.0, 0.0, 0.0};
    bool fin = true;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int p = lane + 32 * k;
        v[0][k] = v[1][k] = v[2][k] = 0.0;
        if (p < N2) {
            const double h = qe[p];
            v[0][k] = a.B[(long)e * N2 + p] + h;
            v[1][k] = qe[p + N2];
            v[2][k] = qe[p + 2 * N2];
            mh = fmin(mh, h);
            fin = fin && isfinite(h) && isfinite(v[1][k]) && isfinite(v[2][k]);
            e2 += v[0][k] * v[0][k];
#pragma unroll
            for (int f = 0; f < 3; ++f) m3[f] += v[f][k];
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int f = 0; f < 3; ++f) m3[f] += __shfl_xor_sync(0xffffffffu, m3[f], off);
        mh = fmin(mh, __shfl_xor_sync(0xffffffffu, mh, off));
        e2 += __shfl_xor_sync(0xffffffffu, e2, off);
    }
    fin = __all_sync(0xffffffffu, fin);
    // deviations from the (double) mean; their statistics in single
    // precision, which is all the BF16 features need
    float dv[3][R], d3[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        m3[f] /= N2;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            dv[f][k] = (lane + 32 * k < N2) ? (float)(v[f][k] - m3[f]) : 0.f;
            d3[f] += dv[f][k] * dv[f][k];
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int f = 0; f < 3; ++f) d3[f] += __shfl_xor_sync(0xffffffffu, d3[f], off);
    __nv_bfloat16* xr = a.X + (long)e * KP;
    float rmsf[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        rmsf[f] = sqrtf(d3[f] * (1.0f / N2));
        const float mf = fabsf((float)m3[f]);
        const float inv = (rmsf[f] > (float)MLP_REL_FLAT * mf && rmsf[f] > 0.0f) ? 1.0f / rmsf[f] : 0.0f;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int p = lane + 32 * k;
            if (p < N2) xr[f * N2 + p] = __float2bfloat16(dv[f][k] * inv);
        }
    }
    if (lane < 3) {  // lanes 0, 1, 2: the scale feature of their field, one log10 pass
        const float r = lane == 0 ? rmsf[0] : (lane == 1 ? rmsf[1] : rmsf[2]);
        const float m = (float)(lane == 0 ? m3[0] : (lane == 1 ? m3[1] : m3[2]));
        const float tot = m * m + r * r;
        const float sf = (tot > 0.0f && r > 0.0f) ? fmaxf(log10f(r * r / tot), (float)MLP_S_MIN) : (float)MLP_S_MIN;
        xr[3 * N2 + lane] = __float2bfloat16(0.25f * sf);
        if (lane == 0) a.seta[e] = sf;
    }
    for (int c = 3 * N2 + 3 + lane; c < KP; c += 32) xr[c] = __float2bfloat16(0.0f);
    if (lane == 0) {
        a.energy[e] = e2;
        a.ok[e] = (fin && mh > a.c.PosPresTOL) ? 1 : 0;
    }
}

// Warps stride over the elements below the live extent (one pass per warp
// with the one-shot grid of a single mesh, a resident grid for an arena).
template <int NGL>
__global__ void __launch_bounds__(256) k_ind_features_warp(IndArgs a) {
    const int lim = a.extent ? min(a.K, a.extent[0]) : a.K;
    for (int e = blockIdx.x * 8 + (threadIdx.x >> 5); e < lim; e += gridDim.x * 8)  // warp-uniform
        ind_features_warp_elem<NGL>(a, e);
}

// The learned decision for one element: 1 when the modal sensor must decide.
__device__ __forceinline__ int learned_needs_modal(const IndArgs& a, double sig, double nodal, int ok) {
    if (!ok) return 1;                                // positivity / finiteness check failed
    if (a.emax * nodal < a.c.ZeroTOL) return 0;       // modal energy below ZeroTOL: sigma = -inf
    if (a.emin * nodal < a.c.ZeroTOL) return 1;       // may be near ZeroTOL
    if (sig < a.c.sigmaMin - a.margin) return 0;
    if (sig > a.c.sigmaMax + a.margin) return 0;
    return 1;
}

// One node's inputs, loaded a tile ahead.
struct IndLoad {
    double h, b;
    int ins;
    int4 nb;
};

template <int NGL>
__device__ __forceinline__ IndLoad ind_load(const IndArgs& a, int t) {
    using S = IndShape<NGL>;
    constexpr int N2 = S::N2;
    const int el = threadIdx.x / N2, nd = threadIdx.x % N2;
    const int e = t * S::NE + el;
    IndLoad L{0.0, 0.0, -1, make_int4(-1, -1, -1, -1)};
    if (e < a.K) {
        L.h = a.q[(long)e * 3 * N2 + nd];
        L.b = a.B[(long)e * N2 + nd];
        L.ins = inst_of(a.elem_inst, e);
        if (nd == 0 && a.act) L.nb = a.nbr[e];
    }
    return L;
}

// The sensor pass (the learned variant after k_ind_features and
// k_mlp_forward).  Persistent: each block walks tiles of NE elements, the
// next tiles' loads in flight while the current one is processed.
template <int NGL, bool LEARNED>
__global__ void __launch_bounds__(IndShape<NGL>::THREADS, 3) k_indicator(IndArgs a, int ntiles) {
    using S = IndShape<NGL>;
    constexpr int N2 = S::N2, NE = S::NE;
    if (a.extent) ntiles = min(ntiles, (a.extent[0] + NE - 1) / NE);
    // an element's nodes form an aligned group of lanes (N2 divides 32)
    constexpr bool GROUP = (32 % N2) == 0;
    __shared__ double sV[N2];
    __shared__ double seta[NE * N2], sM[NE * N2], sW[NE * N2];
    __shared__ int need[NE];
    __shared__ int verdict[NE];  // learned: 0 zero, 1 eps0 (when need == 0)

    const int tid = threadIdx.x;
    const int el = tid / N2, nd = tid % N2;
    const int s = el * N2 + nd;
    if (tid < N2) sV[tid] = a.Vinv[tid];
    unsigned long long cnt[4] = {0, 0, 0, 0};
    constexpr int PF = 2;  // tiles of loads in flight
    int t = blockIdx.x;
    IndLoad ring[PF];
#pragma unroll
    for (int k = 0; k < PF; ++k) {
        const int tk = t + k * gridDim.x;
        ring[k] = (tk < ntiles) ? ind_load<NGL>(a, tk) : IndLoad{};
    }
    for (; t < ntiles; t += gridDim.x) {
        const IndLoad cur = ring[0];
#pragma unroll
        for (int k = 0; k + 1 < PF; ++k) ring[k] = ring[k + 1];
        {
            const int tn = t + PF * gridDim.x;
            ring[PF - 1] = (tn < ntiles) ? ind_load<NGL>(a, tn) : IndLoad{};
        }
        const int e = t * NE + el;
        const bool live = e < a.K && !a.st[cur.ins].done;
        seta[s] = cur.b + cur.h;
        if (nd == 0) {
            int nm = 1, vd = 0;
            if (LEARNED && live) {
                const double sig = (double)a.y[e] + (double)a.seta[e];
                const double nodal = a.energy[e];
                nm = learned_needs_modal(a, sig, nodal, a.ok[e]);
                vd = (nm == 0 && a.emax * nodal >= a.c.ZeroTOL && sig > a.c.sigmaMax + a.margin) ? 1 : 0;
            }
            need[el] = nm;
            verdict[el] = vd;
        }
        // the modal transform where the sensor decides (every element
        // without the network)
        const bool any = LEARNED ? __syncthreads_or(live && nd == 0 && need[el]) : (__syncthreads(), true);
        bool clear = false;
        if (any) {
            const int i = nd / NGL, j = nd % NGL;  // entry (i, j) of M1 and w
            sM[s] = sensor_m1<NGL>(sV, seta + el * N2, i, j);
            __syncthreads();
            sW[s] = sensor_w<NGL>(sV, sM + el * N2, i, j);
            __syncthreads();
            // Screen: energy ratios from sums in any order (shuffles) differ
            // from the reference-order ones by rounding only; far below the
            // 10^sigma_min bound the sensor is exactly zero, so the serial
            // reference-order tail runs only where it can give otherwise.
            if constexpr (GROUP) {
                const double w = sW[s], w2 = w * w;
                constexpr int N = NGL - 1;
                double z1 = ((i == N) || (j == N)) ? w2 : 0.0;
                double z2 = (((i == N - 1) && (j <= N - 1)) || ((j == N - 1) && (i <= N - 1))) ? w2 : 0.0;
                double n1 = w2;
                double n2 = (i < N && j < N) ? w2 : 0.0;
#pragma unroll
                for (int off = N2 / 2; off > 0; off >>= 1) {
                    z1 += __shfl_xor_sync(0xffffffffu, z1, off);
                    z2 += __shfl_xor_sync(0xffffffffu, z2, off);
                    n1 += __shfl_xor_sync(0xffffffffu, n1, off);
                    n2 += __shfl_xor_sync(0xffffffffu, n2, off);
                }
                const double thr = a.c.sensor_skip * (1.0 - 1e-6);
                // both ratios clearly below the bound (NaN compares false)
                clear = n1 > a.c.ZeroTOL * (1.0 + 1e-6) && z1 < thr * n1 && z2 < thr * n2;
                clear = clear || (n1 < a.c.ZeroTOL * (1.0 - 1e-6));  // both ratios are 0 there
            }
        }
        if (live && nd == 0) {
            double v = 0.0;
            int kind = 2;  // 0 net zero, 1 net eps0, 2 modal
            if (need[el]) {
                v = clear ? 0.0 : sensor_tail<NGL>(a.c, sW + el * N2);
            } else {
                kind = verdict[el];
                v = kind ? a.c.eps0 : 0.0;
            }
            a.VP[e] = v;
            if (a.stage0 && v > 0.0) atomicMax(&a.st[cur.ins].visc_key, dbl_key(v));
            // NaN flags too: its viscous path runs as on the full path
            if (a.act && !(v <= 0.0)) mark_active(a.act, e, cur.nb);
            cnt[kind] += 1;
            if (!(v <= 0.0)) cnt[3] += 1;
        }
        __syncthreads();  // shared tiles are rewritten next iteration
    }
    if (a.stats) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (cnt[k]) atomicAdd(&a.stats[k], cnt[k]);
    }
}

// The learned indicator in one pass at n = 4 and n = 5.  The feature pass
// it replaces reduces each element over a butterfly of W lanes (W = 16 at
// n = 4: k_ind_features, one lane per node; W = 32 at n = 5:
// k_ind_features_warp, one warp per element, lanes past the 25th node
// contributing zeros).  Here W / 4 threads hold an element, thread j its
// butterfly slots j, j + W/4, j + W/2, j + 3W/4 (node = slot where the slot
// is a node): the butterfly's two widest levels pair slots inside a thread,
// the rest the element's lanes, so every per-element sum -- means, nodal
// energy, deviations -- and the positivity check are those of the feature
// pass bit for bit.  The modal transform, its screen (n = 4, as in
// k_indicator<4, true>) and the tail follow k_indicator<NGL, true> entry by
// entry.  Each warp runs the network on its own 32 / (W/4) feature rows
// (mlp_warp_forward_rows: a 16-row MMA tile with every row repeated, each
// row's dot products those of k_mlp_forward).  Inside the tile loop no warp
// waits for another; a tile's loads are issued at its start and the other
// resident warps cover their latency.
template <int NGL>
struct FusedShape {
    static constexpr int N2 = NGL * NGL;
    static constexpr int W = N2 <= 16 ? 16 : 32;    // butterfly width of the feature pass
    static constexpr int SLOTS = 4;                 // butterfly slots per thread
    static constexpr int TPE = W / SLOTS;           // threads per element
    static constexpr int EPW = 32 / TPE;            // elements per warp
    static constexpr int THREADS = 256;
    static constexpr int NE = EPW * (THREADS / 32);  // elements per tile
    static constexpr int KP = mlp_kp(NGL);
    static constexpr int XS = KP + 8;               // feature / W1 row stride (bf16), bank-conflict free
    static constexpr int W2S = MLP_H + 8;           // W2 row stride (bf16)
    static constexpr int ES = N2 + 1;               // element stride of the modal arrays (doubles)
    static constexpr bool SCREEN = (32 % N2) == 0;  // k_indicator's any-order screen (aligned lane groups)
    static constexpr bool OK = NGL == 4 || NGL == 5;
};

// Sum over an element's W butterfly slots x[k] (slot j + k W/4 on thread j
// of the element's W/4 lanes), in the order of a W-lane xor butterfly.
template <int TPE, typename T>
__device__ __forceinline__ T slot_sum(const T (&x)[4]) {
    T s = (x[0] + x[2]) + (x[1] + x[3]);
#pragma unroll
    for (int off = TPE / 2; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    return s;
}

template <int NGL>
__global__ void __launch_bounds__(FusedShape<NGL>::THREADS, 3) k_indicator_fused(IndArgs a, int ntiles) {
    using S = FusedShape<NGL>;
    constexpr int N2 = S::N2, NE = S::NE, KP = S::KP, XS = S::XS, W2S = S::W2S, ES = S::ES;
    constexpr int TPE = S::TPE, EPW = S::EPW;
    static_assert(S::OK, "fused indicator: n = 4 or 5");
    if (a.extent) ntiles = min(ntiles, (a.extent[0] + NE - 1) / NE);
    __shared__ __align__(16) __nv_bfloat16 sW1[MLP_H * XS];
    __shared__ __align__(16) __nv_bfloat16 sW2[MLP_H * W2S];
    __shared__ __align__(16) __nv_bfloat16 sX[NE * XS];
    __shared__ __align__(16) float sP32[3 * MLP_H + 4];  // b1, b2, w3, b3
    __shared__ double sV[N2];
    __shared__ double seta[NE * ES], sM[NE * ES], sW[NE * ES];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int el = tid / TPE, j = tid % TPE;
    for (int i = tid; i < N2; i += blockDim.x) sV[i] = a.Vinv[i];
    for (int i = tid; i < MLP_H * KP; i += blockDim.x) sW1[(i / KP) * XS + i % KP] = a.Pb[a.L.w1 + i];
    for (int i = tid; i < MLP_H * MLP_H; i += blockDim.x) sW2[(i / MLP_H) * W2S + i % MLP_H] = a.Pb[a.L.w2 + i];
    for (int i = tid; i < MLP_H; i += blockDim.x) {
        sP32[i] = a.P[a.L.b1 + i];
        sP32[MLP_H + i] = a.P[a.L.b2 + i];
        sP32[2 * MLP_H + i] = a.P[a.L.w3 + i];
    }
    if (tid == 0) sP32[3 * MLP_H] = a.P[a.L.b3];
    __syncthreads();  // the only block barrier: V and the network staged
    double* se = seta + el * ES;
    double* sm = sM + el * ES;
    double* sw = sW + el * ES;
    __nv_bfloat16* xr = sX + el * XS;
    unsigned long long cnt[4] = {0, 0, 0, 0};
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int e = t * NE + el;
        const bool inb = e < a.K;
        // slot k = node j + TPE k: h, eta = b + h, hu, hv.  Slots past the
        // last node hold zeros and mh's start value (as the feature pass's
        // idle lanes); idle elements take h = 1, b = 0, hu = hv = 0.
        double h[4], v0[4], v1[4], v2[4];
        bool val[4];
        int ins = 0;
        int4 nb = make_int4(-1, -1, -1, -1);
        const double* qe = a.q + (long)(inb ? e : 0) * 3 * N2;
        const double* be = a.B + (long)(inb ? e : 0) * N2;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int p = j + TPE * k;
            val[k] = p < N2;
            h[k] = 1.0; v0[k] = 0.0; v1[k] = 0.0; v2[k] = 0.0;
            if (inb && val[k]) {
                h[k] = qe[p];
                v1[k] = qe[p + N2];
                v2[k] = qe[p + 2 * N2];
                v0[k] = be[p] + h[k];
            } else if (val[k]) {
                v0[k] = 0.0 + 1.0;
            }
        }
        if (inb) {
            ins = inst_of(a.elem_inst, e);
            if (j == 0 && a.act) nb = a.nbr[e];
        }
        const bool live = inb && !a.st[ins].done;
        // ---- features (the feature pass) ----
        double e2k[4], mhk[4];
        bool fin = true;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int p = j + TPE * k;
            if (val[k]) se[p] = v0[k];
            e2k[k] = val[k] ? v0[k] * v0[k] : 0.0;
            mhk[k] = val[k] ? h[k] : 1e300;
            fin = fin && (!val[k] || (isfinite(h[k]) && isfinite(v1[k]) && isfinite(v2[k])));
        }
        // the warp-per-element pass (n = 5) starts each lane's sum at 0.0
        // (0.0 + v turns -0.0 into +0.0); the lane-per-node pass sums v
        double m3[3];
        {
            double z0[4], z1[4], z2[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                z0[k] = S::W == 32 ? 0.0 + v0[k] : v0[k];
                z1[k] = S::W == 32 ? 0.0 + v1[k] : v1[k];
                z2[k] = S::W == 32 ? 0.0 + v2[k] : v2[k];
            }
            m3[0] = slot_sum<TPE>(z0);
            m3[1] = slot_sum<TPE>(z1);
            m3[2] = slot_sum<TPE>(z2);
        }
        const double e2 = slot_sum<TPE>(e2k);
        double mh = fmin(fmin(mhk[0], mhk[2]), fmin(mhk[1], mhk[3]));
#pragma unroll
        for (int off = TPE / 2; off > 0; off >>= 1) {
            mh = fmin(mh, __shfl_xor_sync(0xffffffffu, mh, off));
            fin = __shfl_xor_sync(0xffffffffu, (int)fin, off) && fin;
        }
        float rmsf[3];
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            m3[f] /= N2;
            float dv[4], d3[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double v = f == 0 ? v0[k] : (f == 1 ? v1[k] : v2[k]);
                dv[k] = val[k] ? (float)(v - m3[f]) : 0.f;
                d3[k] = dv[k] * dv[k];
            }
            rmsf[f] = sqrtf(slot_sum<TPE>(d3) * (1.0f / N2));
            const float mf = fabsf((float)m3[f]);
            const float inv = (rmsf[f] > (float)MLP_REL_FLAT * mf && rmsf[f] > 0.0f) ? 1.0f / rmsf[f] : 0.0f;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (val[k]) xr[f * N2 + j + TPE * k] = __float2bfloat16(dv[k] * inv);
        }
        float sf = 0.0f;
        if (j < 3) {  // threads 0, 1, 2 of the element: the scale feature of their field
            const float r = j == 0 ? rmsf[0] : (j == 1 ? rmsf[1] : rmsf[2]);
            const float m = (float)(j == 0 ? m3[0] : (j == 1 ? m3[1] : m3[2]));
            const float tot = m * m + r * r;
            sf = (tot > 0.0f && r > 0.0f) ? fmaxf(log10f(r * r / tot), (float)MLP_S_MIN) : (float)MLP_S_MIN;
            xr[3 * N2 + j] = __float2bfloat16(0.25f * sf);
        }
        for (int c = 3 * N2 + 3 + j; c < KP; c += TPE) xr[c] = __float2bfloat16(0.0f);
        const float s_eta = __shfl_sync(0xffffffffu, sf, lane & ~(TPE - 1));
        const int ok = (fin && mh > a.c.PosPresTOL) ? 1 : 0;
        __syncwarp();  // the warp's feature rows complete
        // ---- network (k_mlp_forward) on the warp's rows ----
        const float yw = mlp_warp_forward_rows<KP, EPW, XS, XS, W2S>(sX + warp * EPW * XS, sW1, sW2, sP32);
        const float y = __shfl_sync(0xffffffffu, yw, 4 * (lane / TPE));  // row r's output sits in quad r
        // ---- decision and modal fallback (k_indicator<NGL, true>) ----
        int nm = 1, vd = 0;
        if (live) {
            const double sig = (double)y + (double)s_eta;
            nm = learned_needs_modal(a, sig, e2, ok);
            vd = (nm == 0 && a.emax * e2 >= a.c.ZeroTOL && sig > a.c.sigmaMax + a.margin) ? 1 : 0;
        }
        bool clear = false;
        if (__any_sync(0xffffffffu, live && nm)) {
            // the modal transform, entry by entry as sensor_m1 / sensor_w
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int p = j + TPE * k;
                if (val[k]) sm[p] = sensor_m1<NGL>(sV, se, p / NGL, p % NGL);
            }
            __syncwarp();
            double w[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int p = j + TPE * k;
                w[k] = val[k] ? sensor_w<NGL>(sV, sm, p / NGL, p % NGL) : 0.0;
                if (val[k]) sw[p] = w[k];
            }
            __syncwarp();
            if constexpr (S::SCREEN) {
                constexpr int N = NGL - 1;
                double z1[4], z2[4], n1[4], n2[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int p = j + TPE * k, i = p / NGL, jj = p % NGL;
                    const double w2 = w[k] * w[k];
                    z1[k] = ((i == N) || (jj == N)) ? w2 : 0.0;
                    z2[k] = (((i == N - 1) && (jj <= N - 1)) || ((jj == N - 1) && (i <= N - 1))) ? w2 : 0.0;
                    n1[k] = w2;
                    n2[k] = (i < N && jj < N) ? w2 : 0.0;
                }
                const double Z1 = slot_sum<TPE>(z1), Z2 = slot_sum<TPE>(z2);
                const double N1 = slot_sum<TPE>(n1), N2s = slot_sum<TPE>(n2);
                const double thr = a.c.sensor_skip * (1.0 - 1e-6);
                clear = N1 > a.c.ZeroTOL * (1.0 + 1e-6) && Z1 < thr * N1 && Z2 < thr * N2s;
                clear = clear || (N1 < a.c.ZeroTOL * (1.0 - 1e-6));
            }
        }
        if (live && j == 0) {
            double v = 0.0;
            int kind = 2;  // 0 net zero, 1 net eps0, 2 modal
            if (nm) {
                v = clear ? 0.0 : sensor_tail<NGL>(a.c, sw);
            } else {
                kind = vd;
                v = kind ? a.c.eps0 : 0.0;
            }
            a.VP[e] = v;
            if (a.stage0 && v > 0.0) atomicMax(&a.st[ins].visc_key, dbl_key(v));
            if (a.act && !(v <= 0.0)) mark_active(a.act, e, nb);
            cnt[kind] += 1;
            if (!(v <= 0.0)) cnt[3] += 1;
        }
        __syncwarp();  // the warp's shared rows are rewritten next tile
    }
    if (a.stats) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (cnt[k]) atomicAdd(&a.stats[k], cnt[k]);
    }
}

}  // namespace esdg
