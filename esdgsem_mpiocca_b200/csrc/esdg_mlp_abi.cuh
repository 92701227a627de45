// C ABI of the learned indicator's training kernels (no counterpart in the
// reference).  Every pointer is a device pointer; every call runs on
// `stream` (null: the legacy default stream) and returns without waiting.
// Included at the end of esdg_engine.cu.
#pragma once

#include "esdg_mlp.cuh"

namespace esdg {

static bool mlp_ngl_ok(int ngl) { return ngl >= 3 && ngl <= 6; }

template <int NGL>
static cudaError_t mlp_set_smem() {
    constexpr int KP = mlp_kp(NGL);
    cudaError_t e = cudaFuncSetAttribute(k_mlp_forward<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         MlpSmem<KP>::fwd_bytes(4));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_backward<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 MlpSmem<KP>::bytes(4));
    return e;
}

static int mlp_fail(const std::string& m, int code = ESDG_E_ARG) {
    g_create_error = m;
    return code;
}

static int mlp_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) return ESDG_OK;
    return mlp_fail(std::string(what) + ": " + cudaGetErrorString(e), ESDG_E_CUDA);
}

#define ESDG_MLP_DISPATCH(ngl, CALL) \
    switch (ngl) {                    \
        case 3: CALL(3); break;       \
        case 4: CALL(4); break;       \
        case 5: CALL(5); break;       \
        case 6: CALL(6); break;       \
    }

}  // namespace esdg

extern "C" {

int esdg_mlp_layout(int ngl, int* out8) {
    using namespace esdg;
    if (!mlp_ngl_ok(ngl) || !out8) return mlp_fail("mlp_layout: ngl must be in 3..6 and out8 given");
    const MlpLayout L = mlp_layout(ngl);
    const int v[8] = {L.kp, L.w1, L.b1, L.w2, L.b2, L.w3, L.b3, L.total};
    for (int i = 0; i < 8; ++i) out8[i] = v[i];
    return ESDG_OK;
}

int esdg_mlp_features(int ngl, int K, const double* q, const double* B, const double* Vinv, double ZeroTOL, void* X,
                      float* tgt, float* seta, void* stream) {
    using namespace esdg;
    if (!mlp_ngl_ok(ngl) || K <= 0 || !q || !B || !Vinv || !X) return mlp_fail("mlp_features: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    auto* Xb = (__nv_bfloat16*)X;
#define ESDG_F(NG) k_mlp_features<NG><<<(K + 7) / 8, 256, 0, s>>>(K, q, B, Vinv, ZeroTOL, Xb, tgt, seta)
    ESDG_MLP_DISPATCH(ngl, ESDG_F)
#undef ESDG_F
    return mlp_cuda(cudaSuccess, "mlp_features");
}

int esdg_mlp_cast(int ngl, const float* P, void* Pb, void* stream) {
    using namespace esdg;
    if (!mlp_ngl_ok(ngl) || !P || !Pb) return mlp_fail("mlp_cast: bad arguments");
    const int n = mlp_layout(ngl).total;
    k_mlp_cast<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, P, (__nv_bfloat16*)Pb);
    return mlp_cuda(cudaSuccess, "mlp_cast");
}

int esdg_mlp_forward(int ngl, int M, const void* X, const float* P, const void* Pb, float* y, int blocks,
                     void* stream) {
    using namespace esdg;
    if (!mlp_ngl_ok(ngl) || M <= 0 || !X || !P || !Pb || !y || blocks <= 0)
        return mlp_fail("mlp_forward: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const MlpLayout L = mlp_layout(ngl);
    cudaError_t e = cudaSuccess;
#define ESDG_F(NG)                                                                                          \
    {                                                                                                       \
        constexpr int KP = mlp_kp(NG);                                                                      \
        e = mlp_set_smem<NG>();                                                                             \
        if (e == cudaSuccess)                                                                               \
            k_mlp_forward<KP><<<blocks, 128, MlpSmem<KP>::fwd_bytes(4), s>>>(M, (const __nv_bfloat16*)X, P, \
                                                                         (const __nv_bfloat16*)Pb, y, L); \
    }
    ESDG_MLP_DISPATCH(ngl, ESDG_F)
#undef ESDG_F
    return mlp_cuda(e, "mlp_forward");
}

int esdg_mlp_backward(int ngl, int M, const void* X, const float* tgt, const float* P, const void* Pb,
                      float* partial, int blocks, void* stream) {
    using namespace esdg;
    if (!mlp_ngl_ok(ngl) || M <= 0 || !X || !tgt || !P || !Pb || !partial || blocks <= 0)
        return mlp_fail("mlp_backward: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const MlpLayout L = mlp_layout(ngl);
    cudaError_t e = cudaSuccess;
#define ESDG_F(NG)                                                                                               \
    {                                                                                                            \
        constexpr int KP = mlp_kp(NG);                                                                           \
        e = mlp_set_smem<NG>();                                                                                  \
        if (e == cudaSuccess)                                                                                    \
            k_mlp_backward<KP><<<blocks, 128, MlpSmem<KP>::bytes(4), s>>>(M, (const __nv_bfloat16*)X, tgt, P,    \
                                                                          (const __nv_bfloat16*)Pb, partial, L); \
    }
    ESDG_MLP_DISPATCH(ngl, ESDG_F)
#undef ESDG_F
    return mlp_cuda(e, "mlp_backward");
}

int esdg_mlp_adam(int ngl, int rows, const float* partial, float* G, float* P, void* Pb, float* m, float* v,
                  float lr, float beta1, float beta2, float eps, int step, void* stream) {
    using namespace esdg;
    if (!mlp_ngl_ok(ngl) || rows <= 0 || !partial || !G || !P || !Pb || !m || !v || step < 1)
        return mlp_fail("mlp_adam: bad arguments");
    const MlpLayout L = mlp_layout(ngl);
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    k_mlp_adam<<<(L.total + 255) / 256, 256, 0, (cudaStream_t)stream>>>(L, mlp_nin(ngl), rows, partial, G, P,
                                                                         (__nv_bfloat16*)Pb, m, v, lr, beta1, beta2,
                                                                         eps, c1, c2);
    return mlp_cuda(cudaSuccess, "mlp_adam");
}

}  // extern "C"
