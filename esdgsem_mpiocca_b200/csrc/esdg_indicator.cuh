// Troubled-cell indicator with active-set marking (no counterpart in the
// reference, which evaluates the modal sensor and the whole viscous path
// on every element).
//
// Per element e it writes the artificial viscosity VP[e] and, where
// VP[e] > 0, flags e and its face neighbours in act[] (zeroed before the
// launch).  The viscous terms of an element vanish exactly unless it or a
// neighbour has VP > 0 (the face viscosity is max(VP_L, VP_R), the volume
// term is VP_e times the gradient), so the stage's viscous kernels run on
// the flagged elements only and give the same numbers as on all of them.
//
// LEARNED = false: the modal sensor (shock_sensor, the arithmetic of
// okl/ShockCapturing/ShockCapturing.okl:17-234) on every element.
// LEARNED = true: the MLP (esdg_mlp.cuh) predicts sigma; its answer is
// used only where it is confident -- sigma_hat < sigma_min - margin gives
// VP = 0, sigma_hat > sigma_max + margin gives VP = eps0 -- and the modal
// sensor decides every other element: the ramp band, elements failing the
// positivity check (min h <= PosPresTOL or a non-finite value), and
// elements whose modal energy may be near the sensor's absolute ZeroTOL
// threshold (bounded from the nodal energy by emin/emax).
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
    const int4* __restrict__ side;
    const int4* __restrict__ ftab;
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
};

constexpr int IND_WARPS = 4;  // warps per block, 16 elements per warp

template <int NGL>
struct IndSmem {
    static constexpr int N2 = NGL * NGL, KP = mlp_kp(NGL);
    static constexpr int ETA = 16 * N2 * 8;        // eta (double) per warp
    static constexpr int X = 16 * KP * 2, A1 = 16 * 32 * 2, Z = 16 * 32 * 4, Y = 16 * 4;
    static constexpr int WS = N2 * 8;               // per-lane sensor scratch (16 lanes)
    static constexpr int PER_WARP = ETA + X + A1 + Z + Y + 16 * WS;
    static constexpr int W = MLP_H * KP * 2 + MLP_H * MLP_H * 2;
    static constexpr int V = (N2 * 8 + 255) / 256 * 256;
    static constexpr int bytes(bool learned) { return V + (learned ? W : 0) + IND_WARPS * PER_WARP; }
};

// Flags e and its face neighbours.
__device__ __forceinline__ void mark_active(const IndArgs& a, int e) {
    a.act[e] = 1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int f = a.side[(long)e * 4 + k].x;
        const int4 t = a.ftab[f];
        const int nb = (t.x == e) ? t.y : t.x;
        if (nb >= 0) a.act[nb] = 1;
    }
}

template <int NGL, bool LEARNED>
__global__ void __launch_bounds__(IND_WARPS * 32) k_indicator(IndArgs a) {
    using S = IndSmem<NGL>;
    constexpr int N2 = NGL * NGL, KP = S::KP;
    extern __shared__ __align__(128) unsigned char ind_smem[];
    double* sV = reinterpret_cast<double*>(ind_smem);
    unsigned char* p = ind_smem + S::V;
    __nv_bfloat16* sW1 = reinterpret_cast<__nv_bfloat16*>(p);
    __nv_bfloat16* sW2 = sW1 + MLP_H * KP;
    if (LEARNED) p += S::W;
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    unsigned char* mine = p + w * S::PER_WARP;
    double* seta = reinterpret_cast<double*>(mine);
    __nv_bfloat16* sX = reinterpret_cast<__nv_bfloat16*>(mine + S::ETA);
    __nv_bfloat16* a1b = reinterpret_cast<__nv_bfloat16*>(mine + S::ETA + S::X);
    float* z = reinterpret_cast<float*>(mine + S::ETA + S::X + S::A1);
    float* y16 = reinterpret_cast<float*>(mine + S::ETA + S::X + S::A1 + S::Z);
    double* wsc = reinterpret_cast<double*>(mine + S::ETA + S::X + S::A1 + S::Z + S::Y);
    for (int i = threadIdx.x; i < N2; i += blockDim.x) sV[i] = a.Vinv[i];
    if (LEARNED) mlp_stage_weights(KP, a.Pb, a.L, sW1, sW2);
    __syncthreads();

    const int e0 = (blockIdx.x * IND_WARPS + w) * 16;
    if (e0 >= a.K) return;  // warp-uniform; no block barrier below
    // lane r (< 16) keeps element e0 + r's decision inputs
    bool live = false, need_modal = !LEARNED;
    double my_seta = 0.0, my_E = 0.0, my_minh = 0.0;
    int my_ins = 0;
    for (int r = 0; r < 16; ++r) {
        const int e = e0 + r;
        bool ok = e < a.K;
        int ins = 0;
        if (ok) {
            ins = inst_of(a.elem_inst, e);
            ok = !a.st[ins].done;
        }
        if (lane == r) { live = ok; my_ins = ins; }
        if (!ok) {
            if (LEARNED)
                for (int c = lane; c < KP; c += 32) sX[r * KP + c] = __float2bfloat16(0.0f);
            continue;
        }
        const double* qe = a.q + (long)e * 3 * N2;
        double v[3][(N2 + 31) / 32];
        double mh = 1e300;
        bool fin = true;
#pragma unroll
        for (int k = 0; k < (N2 + 31) / 32; ++k) {
            const int pn = lane + 32 * k;
            v[0][k] = v[1][k] = v[2][k] = 0.0;
            if (pn < N2) {
                const double h = qe[pn];
                const double eta = a.B[(long)e * N2 + pn] + h;
                seta[r * N2 + pn] = eta;
                v[0][k] = eta;
                v[1][k] = qe[pn + N2];
                v[2][k] = qe[pn + 2 * N2];
                mh = fmin(mh, h);
                fin = fin && isfinite(h) && isfinite(v[1][k]) && isfinite(v[2][k]);
            }
        }
        if (LEARNED) {
            double mean, rms, s;
            mlp_field_stats<NGL>(v[0], mean, rms, s);
            const double E = mean * mean + rms * rms;
            const double s_eta = mlp_feature_row<NGL>(v, sX + r * KP);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) mh = fmin(mh, __shfl_xor_sync(0xffffffffu, mh, off));
            fin = __all_sync(0xffffffffu, fin);
            if (lane == r) {
                my_seta = s_eta;
                my_E = E;
                my_minh = fin ? mh : -1e300;  // non-finite: fail the positivity check
            }
        }
    }
    __syncwarp();
    const int e = e0 + lane;
    if (LEARNED) {
        mlp_warp_forward<KP>(sX, sW1, sW2, a.P, a.L, a1b, z, y16);
        if (lane < 16 && live) {
            const double sig = (double)y16[lane] + my_seta;
            const double nodal = my_E * (double)N2;  // sum of eta^2 over the nodes
            if (!(my_minh > a.c.PosPresTOL)) need_modal = true;
            else if (a.emax * nodal < a.c.ZeroTOL) need_modal = false;  // sigma = -inf: no viscosity
            else if (a.emin * nodal < a.c.ZeroTOL) need_modal = true;
            else if (sig < a.c.sigmaMin - a.margin) need_modal = false;
            else if (sig > a.c.sigmaMax + a.margin) need_modal = false;
            else need_modal = true;
        }
    }
    double v = 0.0;
    int kind = 0;  // 0 net zero, 1 net eps0, 2 modal
    if (lane < 16 && live) {
        if (need_modal) {
            v = shock_sensor<NGL>(a.c, seta + lane * N2, sV, wsc + lane * N2);
            kind = 2;
        } else if (LEARNED) {
            const double sig = (double)y16[lane] + my_seta;
            const double nodal = my_E * (double)N2;
            if (a.emax * nodal >= a.c.ZeroTOL && sig > a.c.sigmaMax + a.margin) { v = a.c.eps0; kind = 1; }
        }
        a.VP[e] = v;
        if (a.stage0 && v > 0.0) atomicMax(&a.st[my_ins].visc_key, dbl_key(v));
        if (!(v <= 0.0)) mark_active(a, e);  // NaN flags too: its viscous path must run as on the full path
    }
    if (a.stats) {
        const bool in = lane < 16 && live;
        const unsigned b0 = __ballot_sync(0xffffffffu, in && kind == 0);
        const unsigned b1 = __ballot_sync(0xffffffffu, in && kind == 1);
        const unsigned b2 = __ballot_sync(0xffffffffu, in && kind == 2);
        const unsigned b3 = __ballot_sync(0xffffffffu, in && !(v <= 0.0));
        if (lane == 0) {
            if (b0) atomicAdd(&a.stats[0], (unsigned long long)__popc(b0));
            if (b1) atomicAdd(&a.stats[1], (unsigned long long)__popc(b1));
            if (b2) atomicAdd(&a.stats[2], (unsigned long long)__popc(b2));
            if (b3) atomicAdd(&a.stats[3], (unsigned long long)__popc(b3));
        }
    }
}

}  // namespace esdg
