// Learned troubled-cell indicator: an MLP (F -> 32 -> 32 -> 1, ReLU) on
// per-element features, BF16 weights and activations on the tensor cores
// (warp-level bf16 MMA with FP32 accumulation), FP32 master weights and
// Adam.  It predicts the modal shock sensor's sigma = log10(energy ratio)
// (okl/ShockCapturing/ShockCapturing.okl:131-204).  No counterpart in the
// reference.
//
// Features of one element (row of X, bf16, KP columns, zero padded), for
// the fields f = eta (= h + b, what the sensor sees), hu, hv over the n^2
// nodes:
//   x[f*n^2 + p] = (v_fp - mean_f) / rms_f        (0 when rms_f <= 1e-12 |mean_f|)
//   x[3 n^2 + f] = s_f / 4,  s_f = log10(rms_f^2 / (mean_f^2 + rms_f^2))
//                  clamped to [-12, 0]
// (rms_f is the RMS of the deviation from the mean).  The network output y
// is the scale-free part: sigma_hat = y + s_eta.  Training targets are
// t = clamp(sigma, -12, 0) - s_eta.
//
// The GEMMs are 16-row tiles per warp (K = KP, N = 32): the network's work
// is a few thousand MACs per element, well below the cost of reading the
// element's state, so warp-level MMA suffices; no tile is large enough for
// a CTA-wide tensor-memory pipeline to pay.
#pragma once

#include <cuda_bf16.h>
#include <mma.h>

namespace esdg {

constexpr int MLP_H = 32;
constexpr double MLP_S_MIN = -12.0;
constexpr double MLP_REL_FLAT = 1e-12;  // rms / |mean| below this: no shape features

__host__ __device__ constexpr int mlp_nin(int ngl) { return 3 * ngl * ngl + 3; }
__host__ __device__ constexpr int mlp_kp(int ngl) { return (mlp_nin(ngl) + 15) / 16 * 16; }

// Parameter block (floats): W1[32][KP] (padding columns unused, kept 0),
// b1[32], W2[32][32], b2[32], w3[32], b3, pad to a multiple of 4.
struct MlpLayout {
    int kp, w1, b1, w2, b2, w3, b3, total;
};
__host__ __device__ inline MlpLayout mlp_layout(int ngl) {
    MlpLayout L;
    L.kp = mlp_kp(ngl);
    L.w1 = 0;
    L.b1 = L.w1 + MLP_H * L.kp;
    L.w2 = L.b1 + MLP_H;
    L.b2 = L.w2 + MLP_H * MLP_H;
    L.w3 = L.b2 + MLP_H;
    L.b3 = L.w3 + MLP_H;
    L.total = (L.b3 + 1 + 3) / 4 * 4;
    return L;
}

// Modal sensor value sigma of one element: log10 of the larger of the two
// energy ratios (okl/ShockCapturing/ShockCapturing.okl:131-204), -inf when
// the modal energy n1 is below ZeroTOL (then *tiny is set).  m = nodal
// (h + b) [eta][xi].
template <int NGL>
__device__ double sensor_sigma(double ZeroTOL, const double* m, const double* V, bool* tiny) {
    constexpr int N = NGL - 1;
    double M1[NGL * NGL], w[NGL * NGL];
    for (int i = 0; i < NGL; ++i)
        for (int j = 0; j < NGL; ++j) {
            double acc = 0.0;
            for (int l = 0; l < NGL; ++l) acc += V[i * NGL + l] * m[j * NGL + l];
            M1[i * NGL + j] = acc;
        }
    for (int i = 0; i < NGL; ++i)
        for (int j = 0; j < NGL; ++j) {
            double acc = 0.0;
            for (int l = 0; l < NGL; ++l) acc += M1[i * NGL + l] * V[j * NGL + l];
            w[i * NGL + j] = acc;
        }
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
    const double t1 = (n1 < ZeroTOL) ? 0.0 : z1 / n1;
    const double t2 = (n1 < ZeroTOL) ? 0.0 : z2 / n2s;
    *tiny = n1 < ZeroTOL;
    return log10((t1 < t2) ? t2 : t1);
}

// Normalisation of one field over an element's nodes held by a warp
// (node p = lane + 32 k): mean, RMS of the deviation, and s.
template <int NGL>
__device__ __forceinline__ void mlp_field_stats(const double (&v)[(NGL * NGL + 31) / 32], double& mean, double& rms,
                                                double& s) {
    constexpr int N2 = NGL * NGL, R = (N2 + 31) / 32;
    const int lane = threadIdx.x & 31;
    double a = 0.0;
#pragma unroll
    for (int k = 0; k < R; ++k)
        if (lane + 32 * k < N2) a += v[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
    mean = a / N2;
    double d2 = 0.0;
#pragma unroll
    for (int k = 0; k < R; ++k)
        if (lane + 32 * k < N2) d2 += (v[k] - mean) * (v[k] - mean);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) d2 += __shfl_xor_sync(0xffffffffu, d2, off);
    rms = sqrt(d2 / N2);
    const double tot = mean * mean + rms * rms;
    s = (tot > 0.0 && rms > 0.0) ? fmax(log10(rms * rms / tot), MLP_S_MIN) : MLP_S_MIN;
}

// Writes one element's feature row (bf16, KP columns) from the warp's
// register copy of the element; returns s_eta (all lanes).
template <int NGL>
__device__ __forceinline__ double mlp_feature_row(const double (&v)[3][(NGL * NGL + 31) / 32],
                                                  __nv_bfloat16* __restrict__ xr) {
    constexpr int N2 = NGL * NGL, R = (N2 + 31) / 32, KP = mlp_kp(NGL);
    const int lane = threadIdx.x & 31;
    double s_eta = 0.0;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
        double mean, rms, s;
        mlp_field_stats<NGL>(v[f], mean, rms, s);
        // a deviation at rounding level (constant field) is not a shape
        const double inv = (rms > MLP_REL_FLAT * fabs(mean) && rms > 0.0) ? 1.0 / rms : 0.0;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int p = lane + 32 * k;
            if (p < N2) xr[f * N2 + p] = __float2bfloat16((float)((v[f][k] - mean) * inv));
        }
        if (lane == 0) xr[3 * N2 + f] = __float2bfloat16((float)(0.25 * s));
        if (f == 0) s_eta = s;
    }
    for (int p = 3 * N2 + 3 + lane; p < KP; p += 32) xr[p] = __float2bfloat16(0.0f);
    return s_eta;
}

// Feature rows of every element, and optionally the training target
// t = clamp(sigma, -12, 0) - s_eta (NaN where the modal energy is below
// ZeroTOL: sigma is then set by an absolute threshold that scale-free
// features cannot see) and s_eta.  One warp per element.
template <int NGL>
__global__ void __launch_bounds__(256) k_mlp_features(int K, const double* __restrict__ q, const double* __restrict__ B,
                                                      const double* __restrict__ Vinv, double ZeroTOL,
                                                      __nv_bfloat16* __restrict__ X, float* __restrict__ tgt,
                                                      float* __restrict__ seta) {
    constexpr int N2 = NGL * NGL, R = (N2 + 31) / 32, KP = mlp_kp(NGL);
    __shared__ double sV[N2];
    __shared__ double se[8][N2];
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (threadIdx.x < N2) sV[threadIdx.x] = Vinv[threadIdx.x];
    __syncthreads();
    const int e = blockIdx.x * 8 + w;
    if (e >= K) return;
    const double* qe = q + (long)e * 3 * N2;
    double v[3][R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int p = lane + 32 * k;
        v[0][k] = v[1][k] = v[2][k] = 0.0;
        if (p < N2) {
            v[0][k] = qe[p] + B[(long)e * N2 + p];
            v[1][k] = qe[p + N2];
            v[2][k] = qe[p + 2 * N2];
            se[w][p] = B[(long)e * N2 + p] + qe[p];
        }
    }
    const double s_eta = mlp_feature_row<NGL>(v, X + (long)e * KP);
    if (tgt) {
        __syncwarp();
        if (lane == 0) {
            bool tiny = false;
            const double sg = sensor_sigma<NGL>(ZeroTOL, se[w], sV, &tiny);
            const double c = fmin(fmax(sg, MLP_S_MIN), 0.0);  // -inf -> -12
            tgt[e] = tiny ? __int_as_float(0x7fc00000) : (float)(c - s_eta);
            if (seta) seta[e] = (float)s_eta;
        }
    } else if (seta && lane == 0) {
        seta[e] = (float)s_eta;
    }
}

using namespace nvcuda;

// One warp's forward pass on 16 rows held in shared memory (ld = KP):
// Z1 = X W1^T + b1, A1 = relu(Z1) (bf16), Z2 = A1 W2^T + b2 (float, left
// in z), y = relu(Z2) . w3 + b3 into y16[0..15].
template <int KP>
__device__ __forceinline__ void mlp_warp_forward(const __nv_bfloat16* Xrows, const __nv_bfloat16* W1b,
                                                 const __nv_bfloat16* W2b, const float* __restrict__ P,
                                                 const MlpLayout& L, __nv_bfloat16* a1b, float* z, float* y16) {
    const int lane = threadIdx.x & 31;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2];
    wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa;
    wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::col_major> fb;
#pragma unroll
    for (int n = 0; n < 2; ++n) wmma::fill_fragment(acc[n], 0.0f);
#pragma unroll
    for (int k = 0; k < KP / 16; ++k) {
        wmma::load_matrix_sync(fa, Xrows + k * 16, KP);
#pragma unroll
        for (int n = 0; n < 2; ++n) {
            wmma::load_matrix_sync(fb, W1b + n * 16 * KP + k * 16, KP);  // B(k, n) = W1[n][k]
            wmma::mma_sync(acc[n], fa, fb, acc[n]);
        }
    }
#pragma unroll
    for (int n = 0; n < 2; ++n) wmma::store_matrix_sync(z + n * 16, acc[n], 32, wmma::mem_row_major);
    __syncwarp();
    for (int i = lane; i < 16 * 32; i += 32) a1b[i] = __float2bfloat16(fmaxf(z[i] + P[L.b1 + (i & 31)], 0.0f));
    __syncwarp();
#pragma unroll
    for (int n = 0; n < 2; ++n) wmma::fill_fragment(acc[n], 0.0f);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        wmma::load_matrix_sync(fa, a1b + k * 16, 32);
#pragma unroll
        for (int n = 0; n < 2; ++n) {
            wmma::load_matrix_sync(fb, W2b + n * 16 * 32 + k * 16, 32);
            wmma::mma_sync(acc[n], fa, fb, acc[n]);
        }
    }
#pragma unroll
    for (int n = 0; n < 2; ++n) wmma::store_matrix_sync(z + n * 16, acc[n], 32, wmma::mem_row_major);
    __syncwarp();
    for (int i = lane; i < 16 * 32; i += 32) z[i] += P[L.b2 + (i & 31)];
    __syncwarp();
    if (lane < 16) {
        float s = P[L.b3];
        for (int j = 0; j < 32; ++j) s += fmaxf(z[lane * 32 + j], 0.0f) * P[L.w3 + j];
        y16[lane] = s;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Forward pass on registers: mma.sync.m16n8k16 (BF16 in, FP32 accumulate)
// with the PTX ISA fragment layouts -- lane = 4 g + t; A (16x16, row):
// a0 (g, 2t..2t+1), a1 (g+8, 2t..), a2 (g, 2t+8..), a3 (g+8, 2t+8..);
// B (16x8, col): b0 (k 2t..2t+1, n g), b1 (k 2t+8..2t+9, n g);
// C (16x8): c0,c1 (g, 2t..2t+1), c2,c3 (g+8, 2t..2t+1).  Layer-1 outputs
// of two adjacent n8 tiles form the layer-2 A fragment of one k16 block, so
// bias, ReLU and the BF16 packing stay in registers; the 32 -> 1 layer is a
// per-lane partial dot product reduced over the four lanes of a quad.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned mlp_pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half)
    return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ void mlp_mma16816(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                             unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// The FP32 vectors a lane needs (biases and w3 at its fragment columns
// 8 j + 2 t, 8 j + 2 t + 1), loaded once per warp.
struct MlpLaneParams {
    float b1[8], b2[8], w3[8], b3;
};

__device__ __forceinline__ MlpLaneParams mlp_lane_params(const float* __restrict__ P, const MlpLayout& L) {
    MlpLaneParams r;
    const int t = threadIdx.x & 3;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            r.b1[2 * j + k] = P[L.b1 + 8 * j + 2 * t + k];
            r.b2[2 * j + k] = P[L.b2 + 8 * j + 2 * t + k];
            r.w3[2 * j + k] = P[L.w3 + 8 * j + 2 * t + k];
        }
    r.b3 = P[L.b3];
    return r;
}

// y for the 16 rows of X (bf16, shared, ld KP): lanes with t == 0 hold
// y[g] in y_lo and y[g + 8] in y_hi (every lane of the quad has them).
// W1 [32][KP], W2 [32][32] bf16 in shared memory.
template <int KP>
__device__ __forceinline__ void mlp_warp_forward_regs(const __nv_bfloat16* X, const __nv_bfloat16* W1,
                                                      const __nv_bfloat16* W2, const MlpLaneParams& R,
                                                      float& y_lo, float& y_hi) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const unsigned* Xu = reinterpret_cast<const unsigned*>(X);    // pairs of bf16
    const unsigned* W1u = reinterpret_cast<const unsigned*>(W1);
    const unsigned* W2u = reinterpret_cast<const unsigned*>(W2);
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float b0 = R.b1[2 * j], b1v = R.b1[2 * j + 1];
        acc[j][0] = b0; acc[j][1] = b1v; acc[j][2] = b0; acc[j][3] = b1v;
    }
#pragma unroll
    for (int kb = 0; kb < KP / 16; ++kb) {
        const int c = kb * 8 + t;  // column pair index (2 bf16 per unsigned)
        const unsigned a0 = Xu[g * (KP / 2) + c], a1 = Xu[(g + 8) * (KP / 2) + c];
        const unsigned a2 = Xu[g * (KP / 2) + c + 4], a3 = Xu[(g + 8) * (KP / 2) + c + 4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = 8 * j + g;  // B(k, n) = W1[n][k]
            mlp_mma16816(acc[j], a0, a1, a2, a3, W1u[n * (KP / 2) + c], W1u[n * (KP / 2) + c + 4]);
        }
    }
    float acc2[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float b0 = R.b2[2 * j], b1v = R.b2[2 * j + 1];
        acc2[j][0] = b0; acc2[j][1] = b1v; acc2[j][2] = b0; acc2[j][3] = b1v;
    }
#pragma unroll
    for (int kb = 0; kb < 2; ++kb) {
        // A1 k16 block kb = layer-1 n8 tiles 2 kb and 2 kb + 1, after ReLU
        const int j0 = 2 * kb, j1 = 2 * kb + 1;
        const unsigned a0 = mlp_pack_bf16(fmaxf(acc[j0][0], 0.f), fmaxf(acc[j0][1], 0.f));
        const unsigned a1 = mlp_pack_bf16(fmaxf(acc[j0][2], 0.f), fmaxf(acc[j0][3], 0.f));
        const unsigned a2 = mlp_pack_bf16(fmaxf(acc[j1][0], 0.f), fmaxf(acc[j1][1], 0.f));
        const unsigned a3 = mlp_pack_bf16(fmaxf(acc[j1][2], 0.f), fmaxf(acc[j1][3], 0.f));
        const int c = kb * 8 + t;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = 8 * j + g;  // B(k, n) = W2[n][k]
            mlp_mma16816(acc2[j], a0, a1, a2, a3, W2u[n * 16 + c], W2u[n * 16 + c + 4]);
        }
    }
    float lo = 0.f, hi = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float w0 = R.w3[2 * j], w1 = R.w3[2 * j + 1];
        lo += fmaxf(acc2[j][0], 0.f) * w0 + fmaxf(acc2[j][1], 0.f) * w1;
        hi += fmaxf(acc2[j][2], 0.f) * w0 + fmaxf(acc2[j][3], 0.f) * w1;
    }
    lo += __shfl_xor_sync(0xffffffffu, lo, 1);
    lo += __shfl_xor_sync(0xffffffffu, lo, 2);
    hi += __shfl_xor_sync(0xffffffffu, hi, 1);
    hi += __shfl_xor_sync(0xffffffffu, hi, 2);
    y_lo = lo + R.b3;
    y_hi = hi + R.b3;
}

// The same forward pass for a warp that holds only R rows (R divides 8):
// row r of the 16-row MMA tile is row r % R of X, so a0 = a1 and a2 = a3,
// and every row's dot products are those mlp_warp_forward_regs forms for it
// in a full tile (the same operands, MMAs and FP32 additions, in the same
// order).  Biases and w3 come from shared memory (P32: b1, b2, w3 [32 each],
// b3), so a warp keeps no network parameters in registers between tiles.
// Lane 4 r holds y of row r (r < R).
// Row strides (bf16 elements): XS of X, W1S of W1 [32][W1S], W2S of W2
// [32][W2S]; strides of KP + 8 and 40 keep the fragment loads of a warp free
// of shared-memory bank conflicts.
template <int KP, int R, int XS = KP, int W1S = KP, int W2S = MLP_H>
__device__ __forceinline__ float mlp_warp_forward_rows(const __nv_bfloat16* X, const __nv_bfloat16* W1,
                                                       const __nv_bfloat16* W2, const float* P32) {
    static_assert(8 % R == 0, "rows per warp divide 8");
    static_assert(XS % 8 == 0 && W1S % 8 == 0 && W2S % 8 == 0, "16-byte rows");
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int row = g % R;
    const unsigned* Xu = reinterpret_cast<const unsigned*>(X);
    const unsigned* W1u = reinterpret_cast<const unsigned*>(W1);
    const unsigned* W2u = reinterpret_cast<const unsigned*>(W2);
    const float2* b1 = reinterpret_cast<const float2*>(P32);
    const float2* b2 = reinterpret_cast<const float2*>(P32 + MLP_H);
    const float2* w3 = reinterpret_cast<const float2*>(P32 + 2 * MLP_H);
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float2 b = b1[4 * j + t];
        acc[j][0] = b.x; acc[j][1] = b.y; acc[j][2] = b.x; acc[j][3] = b.y;
    }
#pragma unroll
    for (int kb = 0; kb < KP / 16; ++kb) {
        const int c = kb * 8 + t;
        const unsigned a0 = Xu[row * (XS / 2) + c], a2 = Xu[row * (XS / 2) + c + 4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = 8 * j + g;
            mlp_mma16816(acc[j], a0, a0, a2, a2, W1u[n * (W1S / 2) + c], W1u[n * (W1S / 2) + c + 4]);
        }
    }
    float acc2[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float2 b = b2[4 * j + t];
        acc2[j][0] = b.x; acc2[j][1] = b.y; acc2[j][2] = b.x; acc2[j][3] = b.y;
    }
#pragma unroll
    for (int kb = 0; kb < 2; ++kb) {
        const int j0 = 2 * kb, j1 = 2 * kb + 1;
        const unsigned a0 = mlp_pack_bf16(fmaxf(acc[j0][0], 0.f), fmaxf(acc[j0][1], 0.f));
        const unsigned a2 = mlp_pack_bf16(fmaxf(acc[j1][0], 0.f), fmaxf(acc[j1][1], 0.f));
        const int c = kb * 8 + t;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = 8 * j + g;
            mlp_mma16816(acc2[j], a0, a0, a2, a2, W2u[n * (W2S / 2) + c], W2u[n * (W2S / 2) + c + 4]);
        }
    }
    float lo = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float2 w = w3[4 * j + t];
        lo += fmaxf(acc2[j][0], 0.f) * w.x + fmaxf(acc2[j][1], 0.f) * w.y;
    }
    lo += __shfl_xor_sync(0xffffffffu, lo, 1);
    lo += __shfl_xor_sync(0xffffffffu, lo, 2);
    return lo + P32[3 * MLP_H];
}

// Shared-memory carve-up of the MLP kernels (bytes): the BF16 weights once
// per block, then per warp: X tile, A1 (bf16), Z (float), dZ2 and dZ1
// (bf16), scratch (float), y.
template <int KP>
struct MlpSmem {
    static constexpr int W1 = MLP_H * KP * 2, W2 = MLP_H * MLP_H * 2;
    static constexpr int XW = 16 * KP * 2;
    static constexpr int A1 = 16 * 32 * 2, Z = 16 * 32 * 4, G = 16 * 32 * 2, Y = 16 * 4;
    static constexpr int PER_WARP = XW + A1 + Z + 2 * G + Z + Y;
    static constexpr int bytes(int warps) { return W1 + W2 + warps * PER_WARP; }
    static constexpr int fwd_bytes(int warps) { return W1 + W2 + warps * XW; }
};

__global__ void k_mlp_cast(int n, const float* __restrict__ P, __nv_bfloat16* __restrict__ Pb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) Pb[i] = __float2bfloat16(P[i]);
}

__device__ __forceinline__ void mlp_stage_weights(int KP, const __nv_bfloat16* __restrict__ Pb, const MlpLayout& L,
                                                  __nv_bfloat16* sW1, __nv_bfloat16* sW2) {
    for (int i = threadIdx.x; i < MLP_H * KP; i += blockDim.x) sW1[i] = Pb[L.w1 + i];
    for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) sW2[i] = Pb[L.w2 + i];
}

// Loads 16 rows (rows past M - 1 repeat the last one) into shared memory
// with 16-byte vectors.
template <int KP>
__device__ __forceinline__ void mlp_load_rows(const __nv_bfloat16* __restrict__ X, int M, int r0,
                                              __nv_bfloat16* sX) {
    const int lane = threadIdx.x & 31;
    constexpr int VPR = KP / 8;
    for (int i = lane; i < 16 * VPR; i += 32) {
        const int r = min(r0 + i / VPR, M - 1);
        reinterpret_cast<uint4*>(sX)[i] = reinterpret_cast<const uint4*>(X + (long)r * KP)[i % VPR];
    }
    __syncwarp();
}

// Network output y for M rows.  4 warps per block, grid-stride over 16-row
// tiles; each warp holds its next tile in registers while it evaluates the
// current one.  Dynamic shared memory MlpSmem<KP>::fwd_bytes(4).
template <int KP>
__global__ void __launch_bounds__(128) k_mlp_forward(int M, const __nv_bfloat16* __restrict__ X,
                                                     const float* __restrict__ P,
                                                     const __nv_bfloat16* __restrict__ Pb, float* __restrict__ y,
                                                     MlpLayout L, const int* __restrict__ Mlive = nullptr) {
    if (Mlive) M = min(M, *Mlive);  // rows past a live extent are skipped
    using S = MlpSmem<KP>;
    constexpr int VPR = KP / 8;        // 16-byte vectors per row
    constexpr int NV = 16 * VPR / 32;  // vectors per lane per tile
    extern __shared__ __align__(128) unsigned char mlp_smem[];
    __nv_bfloat16* sW1 = reinterpret_cast<__nv_bfloat16*>(mlp_smem);
    __nv_bfloat16* sW2 = reinterpret_cast<__nv_bfloat16*>(mlp_smem + S::W1);
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    __nv_bfloat16* sX = reinterpret_cast<__nv_bfloat16*>(mlp_smem + S::W1 + S::W2 + w * S::XW);
    mlp_stage_weights(KP, Pb, L, sW1, sW2);
    __syncthreads();
    if (M <= 0) return;
    const int tiles = (M + 15) / 16;
    const int stride = gridDim.x * 4;
    auto fetch = [&](int t, uint4 (&buf)[NV]) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const int i = lane + 32 * k;
            const int r = min(t * 16 + i / VPR, M - 1);
            buf[k] = reinterpret_cast<const uint4*>(X + (long)r * KP)[i % VPR];
        }
    };
    const MlpLaneParams R = mlp_lane_params(P, L);
    uint4 buf[NV];
    int t = blockIdx.x * 4 + w;
    if (t < tiles) fetch(t, buf);
    for (; t < tiles; t += stride) {
#pragma unroll
        for (int k = 0; k < NV; ++k) reinterpret_cast<uint4*>(sX)[lane + 32 * k] = buf[k];
        __syncwarp();
        if (t + stride < tiles) fetch(t + stride, buf);  // in flight during this tile
        float ylo, yhi;
        mlp_warp_forward_regs<KP>(sX, sW1, sW2, R, ylo, yhi);
        const int g = lane >> 2, r0 = t * 16;
        if ((lane & 3) == 0) {
            if (r0 + g < M) y[r0 + g] = ylo;
            if (r0 + g + 8 < M) y[r0 + g + 8] = yhi;
        }
        __syncwarp();  // sX is rewritten next iteration
    }
}

// Gradient of the loss (1/M) sum (y - t)^2 over M rows.  Each warp
// accumulates over its tiles and writes one partial row of L.total floats
// to partial[(blockIdx.x * 4 + warp) * L.total]; slot b3 + 1 of the row
// holds the warp's sum of squared errors.  k_mlp_adam sums the rows in a
// fixed order, so training is deterministic.
template <int KP>
__global__ void __launch_bounds__(128) k_mlp_backward(int M, const __nv_bfloat16* __restrict__ X,
                                                      const float* __restrict__ tgt, const float* __restrict__ P,
                                                      const __nv_bfloat16* __restrict__ Pb,
                                                      float* __restrict__ partial, MlpLayout L) {
    using S = MlpSmem<KP>;
    extern __shared__ __align__(128) unsigned char mlp_smem[];
    __nv_bfloat16* sW1 = reinterpret_cast<__nv_bfloat16*>(mlp_smem);
    __nv_bfloat16* sW2 = reinterpret_cast<__nv_bfloat16*>(mlp_smem + S::W1);
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    unsigned char* mine = mlp_smem + S::W1 + S::W2 + w * S::PER_WARP;
    __nv_bfloat16* sX = reinterpret_cast<__nv_bfloat16*>(mine);
    __nv_bfloat16* a1b = reinterpret_cast<__nv_bfloat16*>(mine + S::XW);
    float* z = reinterpret_cast<float*>(mine + S::XW + S::A1);
    __nv_bfloat16* g2b = reinterpret_cast<__nv_bfloat16*>(mine + S::XW + S::A1 + S::Z);
    __nv_bfloat16* g1b = reinterpret_cast<__nv_bfloat16*>(mine + S::XW + S::A1 + S::Z + S::G);
    float* scr = reinterpret_cast<float*>(mine + S::XW + S::A1 + S::Z + 2 * S::G);
    float* y16 = reinterpret_cast<float*>(mine + S::XW + S::A1 + S::Z + 2 * S::G + S::Z);
    mlp_stage_weights(KP, Pb, L, sW1, sW2);
    __syncthreads();
    const int tiles = (M + 15) / 16;
    const float scale = 2.0f / (float)M;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> gW2[2][2];
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> gW1[2][KP / 16];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
#pragma unroll
        for (int b = 0; b < 2; ++b) wmma::fill_fragment(gW2[a][b], 0.0f);
#pragma unroll
        for (int b = 0; b < KP / 16; ++b) wmma::fill_fragment(gW1[a][b], 0.0f);
    }
    float gb1 = 0.f, gb2 = 0.f, gw3 = 0.f, gb3 = 0.f, l2 = 0.f;  // lane j: column j
    const float w3j = P[L.w3 + lane];
    for (int t = blockIdx.x * 4 + w; t < tiles; t += gridDim.x * 4) {
        const int r0 = t * 16;
        mlp_load_rows<KP>(X, M, r0, sX);
        mlp_warp_forward<KP>(sX, sW1, sW2, P, L, a1b, z, y16);  // z = Z2
        float dy = 0.f;
        if (lane < 16 && r0 + lane < M) {
            const float e = y16[lane] - tgt[r0 + lane];
            dy = scale * e;
            l2 += e * e;
        }
        // dZ2 = dy w3 where Z2 > 0; column sums for b2, w3, b3
        for (int r = 0; r < 16; ++r) {
            const float dyr = __shfl_sync(0xffffffffu, dy, r);
            const float zz = z[r * 32 + lane];
            gw3 += dyr * fmaxf(zz, 0.f);
            const float g = (zz > 0.f) ? dyr * w3j : 0.f;
            gb2 += g;
            g2b[r * 32 + lane] = __float2bfloat16(g);
            gb3 += (lane == 0) ? dyr : 0.f;
        }
        __syncwarp();
        // gW2 += dZ2^T A1: A(m=j, k=r) = dZ2[r][j] (col-major, ld 32), B(k=r, n=i) = A1[r][i] (row-major)
        {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::col_major> fa;
            wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                wmma::load_matrix_sync(fa, g2b + a * 16, 32);
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    wmma::load_matrix_sync(fb, a1b + b * 16, 32);
                    wmma::mma_sync(gW2[a][b], fa, fb, gW2[a][b]);
                }
            }
        }
        // dA1 = dZ2 W2: A = dZ2 (row-major, ld 32), B(k=j, n=i) = W2[j][i] (row-major, ld 32)
        {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa;
            wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb;
            wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2];
#pragma unroll
            for (int n = 0; n < 2; ++n) wmma::fill_fragment(acc[n], 0.f);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                wmma::load_matrix_sync(fa, g2b + k * 16, 32);
#pragma unroll
                for (int n = 0; n < 2; ++n) {
                    wmma::load_matrix_sync(fb, sW2 + k * 16 * 32 + n * 16, 32);
                    wmma::mma_sync(acc[n], fa, fb, acc[n]);
                }
            }
#pragma unroll
            for (int n = 0; n < 2; ++n) wmma::store_matrix_sync(scr + n * 16, acc[n], 32, wmma::mem_row_major);
        }
        __syncwarp();
        // dZ1 = dA1 where A1 > 0
        for (int r = 0; r < 16; ++r) {
            const float g = (__bfloat162float(a1b[r * 32 + lane]) > 0.f) ? scr[r * 32 + lane] : 0.f;
            gb1 += g;
            g1b[r * 32 + lane] = __float2bfloat16(g);
        }
        __syncwarp();
        // gW1 += dZ1^T X: A(m=j, k=r) = dZ1[r][j] (col-major, ld 32), B(k=r, n=c) = X[r][c] (row-major, ld KP)
        {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::col_major> fa;
            wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                wmma::load_matrix_sync(fa, g1b + a * 16, 32);
#pragma unroll
                for (int b = 0; b < KP / 16; ++b) {
                    wmma::load_matrix_sync(fb, sX + b * 16, KP);
                    wmma::mma_sync(gW1[a][b], fa, fb, gW1[a][b]);
                }
            }
        }
        __syncwarp();
    }
    float* out = partial + (long)(blockIdx.x * 4 + w) * L.total;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            wmma::store_matrix_sync(scr, gW2[a][b], 16, wmma::mem_row_major);
            __syncwarp();
            for (int i = lane; i < 256; i += 32) out[L.w2 + (a * 16 + i / 16) * 32 + b * 16 + i % 16] = scr[i];
            __syncwarp();
        }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < KP / 16; ++b) {
            wmma::store_matrix_sync(scr, gW1[a][b], 16, wmma::mem_row_major);
            __syncwarp();
            for (int i = lane; i < 256; i += 32) out[L.w1 + (a * 16 + i / 16) * KP + b * 16 + i % 16] = scr[i];
            __syncwarp();
        }
    out[L.b1 + lane] = gb1;
    out[L.b2 + lane] = gb2;
    out[L.w3 + lane] = gw3;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        l2 += __shfl_xor_sync(0xffffffffu, l2, off);
        gb3 += __shfl_xor_sync(0xffffffffu, gb3, off);
    }
    if (lane == 0) {
        out[L.b3] = gb3;
        out[L.b3 + 1] = l2;
        if (L.b3 + 2 < L.total) out[L.b3 + 2] = 0.f;
        if (L.b3 + 3 < L.total) out[L.b3 + 3] = 0.f;
    }
}

// Sums the R partial rows (fixed order) into G and applies one Adam step
// (Kingma & Ba 2015) to the FP32 master weights, refreshing the BF16 copy;
// c1 = 1 - b1^step, c2 = 1 - b2^step.  Padding columns of W1 and the slots
// past b3 are not updated (slot b3 + 1 of G is the summed squared error).
__global__ void k_mlp_adam(MlpLayout L, int nin, int R, const float* __restrict__ partial, float* __restrict__ G,
                           float* P, __nv_bfloat16* Pb, float* m, float* v, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.total) return;
    float g = 0.f;
    for (int r = 0; r < R; ++r) g += partial[(long)r * L.total + i];
    G[i] = g;
    const bool pad = (i < L.b1 && (i % L.kp) >= nin) || i > L.b3;
    if (pad) return;
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float p = P[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    P[i] = p;
    Pb[i] = __float2bfloat16(p);
}

}  // namespace esdg
