// Batched ensemble ("arena") of independent instances of one polynomial
// degree advanced together: every kernel launch of a step covers all
// instances, each with its own time, time step (own CFL reduction), end
// time and step cap.  No counterpart in the reference (it runs one mesh per
// process).
//
// Device layout: element and face arrays of fixed capacity (K_cap, F_cap);
// an instance occupies a contiguous element range and a contiguous face
// range (its own numbering shifted by the range starts).  elem_inst[e]
// names the owner of element e; unused elements belong to a retired slot
// whose step state has done = 1, so every kernel skips them.  The step is
// captured once into a CUDA graph over the whole capacity and stays valid
// while instances are added and removed between replays, which is what
// continuous batching needs.
#pragma once

#include <algorithm>
#include <map>
#include <vector>

namespace esdg {

// Fills n entries with a value (element-to-instance map).
__global__ void k_fill_int(int* p, long n, int v) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

class Arena : public Engine {
  public:
    struct Range {
        int begin, size;
    };
    struct Inst {
        bool live = false;
        Range e{0, 0}, f{0, 0};
        int K = 0, F = 0;
    };
    int max_inst = 0, K_cap = 0, F_cap = 0;
    std::vector<Inst> inst;
    std::vector<Range> free_e, free_f;
    std::vector<DevState> st_h;  // host copy of all step states (pinned not needed: small)
    double* dAv = nullptr;       // staging for per-instance uploads (host)

    static bool take(std::vector<Range>& fl, int n, Range* out) {
        for (size_t k = 0; k < fl.size(); ++k)
            if (fl[k].size >= n) {
                *out = {fl[k].begin, n};
                fl[k].begin += n;
                fl[k].size -= n;
                if (fl[k].size == 0) fl.erase(fl.begin() + k);
                return true;
            }
        return false;
    }
    static void give(std::vector<Range>& fl, Range r) {
        if (r.size <= 0) return;
        fl.push_back(r);
        std::sort(fl.begin(), fl.end(), [](const Range& a, const Range& b) { return a.begin < b.begin; });
        std::vector<Range> m;
        for (auto& x : fl) {
            if (!m.empty() && m.back().begin + m.back().size == x.begin) m.back().size += x.size;
            else m.push_back(x);
        }
        fl.swap(m);
    }

    int create(int N_, int maxI, int Kc, int Fc, int NumFlux_, int ES_, double g_, double tol, int AV_, double eps0_,
               double smax, double smin, int PP_, int rkOrder, int rkSSP_) {
        if (maxI <= 0 || Kc <= 0 || Fc <= 0) return fail(ESDG_E_ARG, "arena: capacities must be positive");
        Basis B;
        if (N_ < 1 || N_ > 7) return fail(ESDG_E_UNSUPPORTED, "N must be in 1..7");
        build_basis(N_, 1, &B);
        // element Kc is a sentinel owned by the retired slot (target of unused
        // face entries); the allocation is kept even for the bulk copies
        const int Ka = (Kc + 1) % 2 ? Kc + 2 : Kc + 1;
        I = maxI + 1;  // slot maxI: retired (done) owner of unused elements
        int r = init(N_, Ka, Fc, 0, rkSSP_, ES_, 0, eps0_, smax, smin, tol, 1.0 / B.wGL[0], g_, PP_, AV_, 0, 0.0, 0, 0);
        if (r) return r;
        max_inst = maxI;
        K_cap = Kc;
        F_cap = Fc;
        if ((r = alloc(&elem_inst, (size_t)Ka)) || (r = alloc(&extent, 2))) return r;  // extent {0, 0}: none live
        st_h.assign(I, DevState{});
        for (auto& s : st_h) { std::memset(&s, 0, sizeof s); s.done = 1; s.T = 0; }
        cudaError_t e = cudaMemcpy(st, st_h.data(), sizeof(DevState) * I, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "arena state upload");
        k_fill_int<<<(Ka + 255) / 256, 256>>>(elem_inst, Ka, maxI);
        // unused element sides point at face 0, unused faces at the sentinel
        std::vector<int4> side0((size_t)Ka * 4, make_int4(0, 1, 1, 0));
        std::vector<int4> face0((size_t)Fc, make_int4(Kc, -1, 0, 0));
        e = cudaMemcpy(side, side0.data(), side0.size() * sizeof(int4), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(ftab, face0.data(), face0.size() * sizeof(int4), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return cuda_fail(e, "arena tables");
        // global operators
        if ((r = h2d(D, B.D.data(), B.D.size(), "D")) || (r = h2d(Dstrong, B.Dstrong.data(), B.Dstrong.size(), "Ds")) ||
            (r = h2d(Dhat, B.Dhat.data(), B.Dhat.size(), "Dhat")) ||
            (r = h2d(Vinv, B.VdmInv.data(), B.VdmInv.size(), "Vinv")) ||
            (r = h2d(GLw, B.wGL.data(), B.wGL.size(), "GLw")))
            return r;
        Vinv_h = B.VdmInv;
        Dfd_h = B.D;
        copied = true;
        if ((r = build(1, NumFlux_, rkSSP_, AV_, PP_, 0, 0))) return r;
        double A[8], Bc[8], C[8];
        const int s = rk_coefficients(rkOrder, rkSSP_, A, Bc, C);
        if (!s) return fail(ESDG_E_UNSUPPORTED, "RK order must be 3 or 4");
        gA.assign(A, A + s); gB.assign(Bc, Bc + s); gC.assign(C, C + s);
        gStages = s;
        inst.assign(maxI, Inst{});
        free_e = {{0, Kc}};
        free_f = {{0, Fc}};
        return capture_step_graph();
    }

    // Adds one instance; its arrays are in its own numbering (as for
    // copyDeviceVariables).  Returns the slot id in *id.
    int add(int K_, int F_, const double* nx_h, const double* ny_h, const double* scal_h, const double* yxi_h,
            const double* yeta_h, const double* xxi_h, const double* xeta_h, const double* b_h, const double* Bx_h,
            const double* By_h, const double* J_h, const double* q_h, const double* Es_h, const int* MS_h,
            const int* OR_h, const int* E2E_h, const int* ED_h, double T_, int max_steps_, double minEle,
            double CFL_, double DFL_, int* id) {
        if (!id) return fail(ESDG_E_ARG, "null id");
        int slot = -1;
        for (int k = 0; k < max_inst; ++k)
            if (!inst[k].live) { slot = k; break; }
        if (slot < 0) return fail(ESDG_E_NOMEM, "arena: no free instance slot");
        Range re, rf;
        if (!take(free_e, K_, &re)) return fail(ESDG_E_NOMEM, "arena: no contiguous element range free");
        if (!take(free_f, F_, &rf)) { give(free_e, re); return fail(ESDG_E_NOMEM, "arena: no contiguous face range free"); }
        const int n2 = ngl * ngl;
        const size_t nn = (size_t)K_ * n2, nf = (size_t)F_ * ngl;
        // connectivity in arena numbering, validated
        std::vector<int4> ft(F_), sd((size_t)K_ * 4);
        std::vector<int> ed((size_t)F_ * 8);
        auto bad = [&](const char* m) { give(free_e, re); give(free_f, rf); return fail(ESDG_E_ARG, m); };
        for (int f = 0; f < F_; ++f) {
            const int* r = ED_h + (size_t)f * 8;
            const int eL = r[0], eR = r[1], sL = r[2], sR = r[3], same = r[4] ? 1 : 0;
            if (eL < 0 || eL >= K_ || sL < 0 || sL > 3 || r[5] != 0) return bad("EdgeData: bad left element/side");
            int* o = &ed[(size_t)f * 8];
            o[0] = eL + re.begin; o[2] = sL; o[4] = same; o[5] = 0; o[7] = f + rf.begin;
            if (r[6] == -1) {
                o[1] = -1; o[3] = -1; o[6] = -1;
                ft[f] = make_int4(eL + re.begin, -1, sL | (same << 4), 0);
            } else {
                if (r[6] != 0 || eR < 0 || eR >= K_ || sR < 0 || sR > 3) return bad("EdgeData: bad right element/side");
                o[1] = eR + re.begin; o[3] = sR; o[6] = 0;
                ft[f] = make_int4(eL + re.begin, eR + re.begin, sL | (sR << 2) | (same << 4), 0);
            }
        }
        for (int e = 0; e < K_; ++e)
            for (int s = 0; s < 4; ++s) {
                const size_t k = (size_t)e * 4 + s;
                const int fc = E2E_h[k] - 1;
                if (fc < 0 || fc >= F_ || (MS_h[k] != 1 && MS_h[k] != -1) || (OR_h[k] != 0 && OR_h[k] != 1))
                    return bad("element tables out of range");
                sd[k] = make_int4(fc + rf.begin, MS_h[k], OR_h[k], 0);
            }
        if (pack_face_flags(ft, sd, re.begin, rf.begin)) {
            give(free_e, re); give(free_f, rf);
            return ESDG_E_ARG;
        }
        const size_t eo = (size_t)re.begin, fo = (size_t)rf.begin;
        int r = 0;
        if ((r = h2d(nx + fo * ngl, nx_h, nf, "nx")) || (r = h2d(ny + fo * ngl, ny_h, nf, "ny")) ||
            (r = h2d(scal + fo * ngl, scal_h, nf, "scal")) || (r = h2d(Yxi + eo * n2, yxi_h, nn, "y_xi")) ||
            (r = h2d(Yeta + eo * n2, yeta_h, nn, "y_eta")) || (r = h2d(Xxi + eo * n2, xxi_h, nn, "x_xi")) ||
            (r = h2d(Xeta + eo * n2, xeta_h, nn, "x_eta")) || (r = h2d(B + eo * n2, b_h, nn, "b")) ||
            (r = h2d(Bx + eo * n2, Bx_h, nn, "Bx")) || (r = h2d(By + eo * n2, By_h, nn, "By")) ||
            (r = h2d(Jinv + eo * n2, J_h, nn, "Jinv")) || (r = h2d(q + eo * n2 * 3, q_h, nn * 3, "q")) ||
            (r = h2d(EleSizes + eo, Es_h, (size_t)K_, "EleSizes")) ||
            (r = h2d(ftab + fo, ft.data(), (size_t)F_, "faces")) || (r = h2d(side + eo * 4, sd.data(), sd.size(), "sides")) ||
            (r = h2d(EdgeData + fo * 8, ed.data(), ed.size(), "EdgeData"))) {
            give(free_e, re); give(free_f, rf);
            return r;
        }
        cudaMemsetAsync(gRK + eo * n2 * 3, 0, nn * 3 * sizeof(double), stream);
        // step state, owner map, bathymetry traces, initial wave speed
        DevState s0;
        std::memset(&s0, 0, sizeof s0);
        s0.T = T_; s0.minEle = minEle; s0.CFL = CFL_; s0.DFL = DFL_; s0.max_steps = max_steps_;
        st_h[slot] = s0;
        cudaMemcpyAsync(st + slot, &st_h[slot], sizeof(DevState), cudaMemcpyHostToDevice, stream);
        k_fill_int<<<(K_ + 255) / 256, 256, 0, stream>>>(elem_inst + eo, K_, slot);
        k_collect_bottom_impl<<<(F_ * ngl + 255) / 256, 256, 0, stream>>>(F_, ngl, EdgeData + fo * 8, B, bL + fo * ngl,
                                                                          bR + fo * ngl);
        ranged_lambda(re);
        if (nbr) k_build_nbr<<<(K_ + 255) / 256, 256, 0, stream>>>(re.begin, K_, side, ftab, nbr);
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "arena add");
        inst[slot].live = true;
        inst[slot].e = re;
        inst[slot].f = rf;
        inst[slot].K = K_;
        inst[slot].F = F_;
        *id = slot;
        return update_extent();
    }

    // Highest live element and face (+1), read by the main kernels so that a
    // sparsely filled arena costs what its live part costs.
    int ext_h[2] = {0, 0};
    int update_extent() {
        int ke = 0, kf = 0;
        for (auto& x : inst)
            if (x.live) {
                ke = std::max(ke, x.e.begin + x.e.size);
                kf = std::max(kf, x.f.begin + x.f.size);
            }
        ext_h[0] = ke;
        ext_h[1] = kf;
        cudaError_t e = cudaMemcpyAsync(extent, ext_h, sizeof(ext_h), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "arena extent");
        return 0;
    }

    template <int NGL>
    void lambda_range(Range re) {
        using S = ElemShape<NGL>;
        const long n2 = NGL * NGL;
        k_lambda<NGL><<<(re.size + S::NE - 1) / S::NE, S::THREADS, 0, stream>>>(
            re.size, q + re.begin * n2 * 3, elem_inst + re.begin, st, phys());
    }
    void ranged_lambda(Range re) {
        switch (ngl) {
            case 2: lambda_range<2>(re); break;
            case 3: lambda_range<3>(re); break;
            case 4: lambda_range<4>(re); break;
            case 5: lambda_range<5>(re); break;
            case 6: lambda_range<6>(re); break;
            case 7: lambda_range<7>(re); break;
            case 8: lambda_range<8>(re); break;
        }
    }

    int remove(int id) {
        if (id < 0 || id >= max_inst || !inst[id].live) return fail(ESDG_E_ARG, "arena: no such live instance");
        Inst& in = inst[id];
        k_fill_int<<<(in.K + 255) / 256, 256, 0, stream>>>(elem_inst + in.e.begin, in.K, max_inst);
        std::vector<int4> face0((size_t)in.F, make_int4(K_cap, -1, 0, 0));
        cudaMemcpyAsync(ftab + in.f.begin, face0.data(), face0.size() * sizeof(int4), cudaMemcpyHostToDevice, stream);
        st_h[id].done = 1;
        cudaMemcpyAsync(&st[id].done, &st_h[id].done, sizeof(int), cudaMemcpyHostToDevice, stream);
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "arena remove");
        give(free_e, in.e);
        give(free_f, in.f);
        in = Inst{};
        return update_extent();
    }

    int poll_all() {
        cudaError_t e = cudaMemcpyAsync(st_h.data(), st, sizeof(DevState) * I, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "arena state read-back");
        return 0;
    }

    int advance_arena(int nsteps) {
        int r = launch_arena(nsteps);
        return r ? r : poll_all();
    }

    // Replays the step graph nsteps times without waiting.
    int launch_arena(int nsteps) {
        if (!tma_tuned && ext_h[0] > 0) {
            // tune on the first live contents, then re-capture with the choice
            const int before = tma_variant;
            tune_K = ext_h[0];
            int r = run_autotune();
            if (r) return r;
            if (tma_variant != before && (r = capture_step_graph())) return r;
        }
        for (int k = 0; k < nsteps; ++k) {
            cudaError_t e = cudaGraphLaunch(graph, stream);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
            launches += kernels_per_step;
        }
        return 0;
    }

    int copy_q_inst(int id, double* qh) {
        if (id < 0 || id >= max_inst || !inst[id].live || !qh) return fail(ESDG_E_ARG, "arena: no such live instance");
        const size_t n2 = (size_t)ngl * ngl;
        cudaError_t e = cudaMemcpyAsync(qh, q + inst[id].e.begin * n2 * 3, (size_t)inst[id].K * n2 * 3 * sizeof(double),
                                        cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e, "arena copy q");
        return 0;
    }
};

}  // namespace esdg

struct esdg_ensemble {
    esdg::Arena a;
};

extern "C" {

int esdg_ensemble_create(int device_id, int N, int max_instances, int K_capacity, int F_capacity, int NumFlux, int ES,
                         double g_const, double PosPresTOL, int ArtificialViscosity, double epsilon_0,
                         double sigma_max, double sigma_min, int PositivityPreserving, int rkOrder, int rkSSP,
                         esdg_ensemble** out) {
    if (!out) return ESDG_E_ARG;
    *out = nullptr;
    int dev = device_id;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return ESDG_E_CUDA;
    if (cudaSetDevice(dev) != cudaSuccess) return ESDG_E_CUDA;
    esdg_ensemble* en = new (std::nothrow) esdg_ensemble();
    if (!en) return ESDG_E_NOMEM;
    en->a.device = dev;
    cudaError_t e = cudaStreamCreateWithFlags(&en->a.own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete en; return ESDG_E_CUDA; }
    en->a.stream = en->a.own_stream;
    const int r = en->a.create(N, max_instances, K_capacity, F_capacity, NumFlux, ES, g_const, PosPresTOL,
                               ArtificialViscosity, epsilon_0, sigma_max, sigma_min, PositivityPreserving, rkOrder,
                               rkSSP);
    if (r) {
        esdg::g_create_error = en->a.err;
        en->a.release();
        cudaStreamDestroy(en->a.own_stream);
        delete en;
        return r;
    }
    *out = en;
    return ESDG_OK;
}

int esdg_ensemble_add(esdg_ensemble* en, int Nelem, int Nfaces, const double* normalsX, const double* normalsY,
                      const double* Scal, const double* y_xi, const double* y_eta, const double* x_xi,
                      const double* x_eta, const double* b, const double* Bx, const double* By, const double* J,
                      const double* q, const double* ElementSizes, const int* ElemEdgeMasterSlave,
                      const int* ElemEdgeOrientation, const int* ElemToEdge, const int* EdgeData, double T,
                      int max_steps, double minEleSize, double CFL, double DFL, int* id) {
    if (!en) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    if (!normalsX || !normalsY || !Scal || !y_xi || !y_eta || !x_xi || !x_eta || !b || !Bx || !By || !J || !q ||
        !ElementSizes || !ElemEdgeMasterSlave || !ElemEdgeOrientation || !ElemToEdge || !EdgeData || Nelem <= 0 ||
        Nfaces <= 0)
        return en->a.fail(ESDG_E_ARG, "ensemble_add: every array and positive sizes are required");
    return en->a.add(Nelem, Nfaces, normalsX, normalsY, Scal, y_xi, y_eta, x_xi, x_eta, b, Bx, By, J, q, ElementSizes,
                     ElemEdgeMasterSlave, ElemEdgeOrientation, ElemToEdge, EdgeData, T, max_steps, minEleSize, CFL,
                     DFL, id);
}

int esdg_ensemble_remove(esdg_ensemble* en, int id) {
    if (!en) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    return en->a.remove(id);
}

int esdg_ensemble_advance(esdg_ensemble* en, int nsteps) {
    if (!en || nsteps < 0) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    return en->a.advance_arena(nsteps);
}

int esdg_ensemble_launch(esdg_ensemble* en, int nsteps) {
    if (!en || nsteps < 0) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    return en->a.launch_arena(nsteps);
}

int esdg_ensemble_sync(esdg_ensemble* en) {
    if (!en) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    return en->a.poll_all();
}

int esdg_ensemble_status(esdg_ensemble* en, int id, double* t, int* steps, int* done, int* status) {
    if (!en || id < 0 || id >= en->a.max_inst) return ESDG_E_ARG;
    const esdg::DevState& s = en->a.st_h[id];
    if (t) *t = s.t;
    if (steps) *steps = s.steps;
    if (done) *done = s.done;
    if (status) *status = s.status;
    return ESDG_OK;
}

int esdg_ensemble_copy_q(esdg_ensemble* en, int id, double* q) {
    if (!en) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    return en->a.copy_q_inst(id, q);
}

int esdg_ensemble_free_capacity(const esdg_ensemble* en, int* K_largest, int* F_largest, int* free_slots) {
    if (!en) return ESDG_E_ARG;
    int ke = 0, kf = 0, fs = 0;
    for (auto& r : en->a.free_e) ke = std::max(ke, r.size);
    for (auto& r : en->a.free_f) kf = std::max(kf, r.size);
    for (auto& in : en->a.inst) fs += in.live ? 0 : 1;
    if (K_largest) *K_largest = ke;
    if (F_largest) *F_largest = kf;
    if (free_slots) *free_slots = fs;
    return ESDG_OK;
}

long long esdg_ensemble_bytes(const esdg_ensemble* en) { return en ? (long long)en->a.bytes : -1; }

long long esdg_ensemble_kernel_launches(const esdg_ensemble* en) { return en ? en->a.launches : -1; }

int esdg_ensemble_set_stream(esdg_ensemble* en, void* cuda_stream) {
    if (!en) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    en->a.stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : en->a.own_stream;
    return en->a.capture_step_graph();
}

int esdg_ensemble_set_element_variant(esdg_ensemble* en, int variant) {
    if (!en) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    return en->a.set_element_variant(variant);
}

int esdg_ensemble_element_variants(const esdg_ensemble* en, int* chosen, int* count, float* ms, int* ctas_per_sm,
                                   int cap) {
    if (!en) return ESDG_E_ARG;
    return element_variants(en->a, chosen, count, ms, ctas_per_sm, cap);
}

int esdg_ensemble_set_indicator(esdg_ensemble* en, int mode, const float* params, int nparams, float margin) {
    if (!en) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    return en->a.set_indicator(mode, params, nparams, margin);
}

int esdg_ensemble_set_indicator_every_stage(esdg_ensemble* en, int every_stage) {
    if (!en) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    return en->a.set_indicator_every_stage(every_stage);
}

int esdg_ensemble_indicator_stats(esdg_ensemble* en, unsigned long long* counts4, int reset) {
    if (!en || !counts4) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    return en->a.indicator_stats(counts4, reset);
}

const char* esdg_ensemble_last_error(const esdg_ensemble* en) {
    return en ? en->a.err.c_str() : esdg::g_create_error.c_str();
}

int esdg_ensemble_destroy(esdg_ensemble* en) {
    if (!en) return ESDG_E_ARG;
    cudaSetDevice(en->a.device);
    en->a.release();
    if (en->a.own_stream) cudaStreamDestroy(en->a.own_stream);
    delete en;
    return ESDG_OK;
}

}  // extern "C"
