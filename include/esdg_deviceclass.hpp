// esdg_deviceclass.hpp -- C++ drop-in for the reference's `deviceclass`
// (include/deviceclass.h:28-138 of ESDGSEM_MPIOCCA), forwarding to the C ABI
// of esdg_b200.h.  Same class name, constructor, member functions, argument
// lists and public members that main.cpp uses (`device.bytesAllocated()`,
// `o_q.copyTo(q)`).  DGtimeloop takes the reference's MPI_setup /
// MeshPartitioning / RungeKutta / basis / SW2D objects as template parameters
// and reads from them only what the time loop needs (RK.rkStages and its
// coefficient tables), so this header has no dependency on the reference.
//
// Errors: the reference aborts inside OCCA or throws; this facade throws
// std::runtime_error carrying the engine's status code and message.
#pragma once

#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "esdg_b200.h"

namespace esdg_dropin {

// Tecplot writers of the time loop's outputs, in the file format of the
// reference's src/Plots.cpp (file names under movie/, titles, variable
// lists, one POINT zone of ngl x ngl per element, default stream
// formatting), so that its post-processing reads them unchanged.
namespace tecplot {

inline std::ofstream open(const std::string& name) {
    std::ofstream f(name.c_str());
    if (!f) throw std::runtime_error("esdg plot: cannot open " + name + " (is there a movie/ directory?)");
    return f;
}

// src/Plots.cpp:20-107 (PlotVar 1: H = h + b; PlotVar 2: free surface
// h + b - h_0 and bottom b - h_0; PlotVar 0: no file).
inline void solution(int K, int ngl, int PlotVar, const double* x, const double* y, const double* Q, const double* b,
                     int plotCount, double h0) {
    if (PlotVar != 1 && PlotVar != 2) return;
    std::ostringstream os;
    os << "movie/plot_" << plotCount << ".tec";
    std::ofstream f = open(os.str());
    const int n2 = ngl * ngl;
    f << "TITLE = H_solution.tec\n";
    f << (PlotVar == 1 ? "VARIABLES = \"x\",\"y\",\"H\",\"hu\",\"hv\",\"bottom\"\n"
                       : "VARIABLES = \"x\",\"y\",\"FreeSurface\",\"hu\",\"hv\",\"bottom\"\n");
    for (int ie = 0; ie < K; ie++) {
        f << "ZONE I =" << ngl << ",J=" << ngl << ",F=POINT\n";
        for (int j = 0; j < ngl; ++j)
            for (int i = 0; i < ngl; ++i) {
                const long id = (long)ie * n2 * 3 + j * ngl + i, xid = (long)ie * n2 + j * ngl + i;
                const double H = PlotVar == 1 ? Q[id] + b[xid] : Q[id] + b[xid] - h0;
                const double bottom = PlotVar == 1 ? b[xid] : b[xid] - h0;
                f << x[xid] << " " << y[xid] << " " << H << " " << Q[id + n2] << " " << Q[id + 2 * n2] << " "
                  << bottom << " \n";
            }
    }
}

// src/Plots.cpp:349-399: the element viscosity as a per-node field.
inline void viscosity(int K, int ngl, const double* x, const double* y, const double* eps, int plotCount) {
    std::ostringstream os;
    os << "movie/visc_" << plotCount << ".tec";
    std::ofstream f = open(os.str());
    f << "TITLE = ArtVisc.tec\n";
    f << "VARIABLES = \"x\",\"y\",\"Eps\"\n";
    for (int ie = 0; ie < K; ie++) {
        f << "ZONE I =" << ngl << ",J=" << ngl << ",F=POINT\n";
        for (int j = 0; j < ngl; ++j)
            for (int i = 0; i < ngl; ++i) {
                const long xid = (long)ie * ngl * ngl + j * ngl + i;
                f << x[xid] << " " << y[xid] << " " << eps[ie] << " \n";
            }
    }
    f << "Test";
}

// src/Plots.cpp:151-231: one nodal field (arrival times, maximum elevation).
inline void nodal(const char* file, const char* title, const char* var, int K, int ngl, const double* x,
                  const double* y, const double* v) {
    std::ofstream f = open(std::string("movie/") + file);
    f << "TITLE = " << title << "\n";
    f << "VARIABLES = \"x\",\"y\",\"" << var << "\",\n";
    for (int ie = 0; ie < K; ie++) {
        f << "ZONE I =" << ngl << ",J=" << ngl << ",F=POINT\n";
        for (int j = 0; j < ngl; ++j)
            for (int i = 0; i < ngl; ++i) {
                const long xid = (long)ie * ngl * ngl + j * ngl + i;
                f << x[xid] << " " << y[xid] << " " << v[xid] << " \n";
            }
    }
}

// src/Plots.cpp:401-476: total entropy and relative mass change over time.
inline void entropy(int n, const double* t, const double* S) {
    std::ofstream f = open("movie/Entropyplot.tec");
    f << "TITLE = Entropyplot.tec\n";
    f << "VARIABLES = \"t\",\"Entropy\"\n";
    for (int i = 0; i < n; ++i) f << t[i] << " " << S[i] << " \n";
}
inline void mass(int n, const double* t, const double* M) {
    std::ofstream f = open("movie/Massplot.tec");
    f << "TITLE = Massplot.tec\n";
    f << "VARIABLES = \"t\",\"Massdifference\"\n";
    for (int i = 0; i < n; ++i) f << t[i] << " " << (M[i] - M[0]) / M[0] << " \n";
}

// src/Plots.cpp:478-517: the seven tide-gauge series.
inline void gauges(int n, const double* t, const std::vector<double> (&g)[7]) {
    std::ofstream f = open("movie/Timeseries.tec");
    f << "TITLE = Timeseries.tec\n";
    f << "VARIABLES = \"t\",\"Chennai\",\"Tuticorin\",\"Visakhapatnam\",\"Paradip\",\"Kochi\",\"Mormugao\","
         "\"Okha\"\n";
    for (int i = 0; i < n; ++i) {
        f << t[i];
        for (int k = 0; k < 7; ++k) f << " " << g[k][i];
        f << " \n";
    }
}

}  // namespace tecplot

// Plot checkpoints of DGtimeloop (src/deviceclass.cpp:711-785): NumPlots
// equidistant times on [0, T] and the fixed lists of some test cases.
inline std::vector<double> plot_checkpoints(int& NumPlots, int Testcase, double T) {
    if (NumPlots <= 0) return {};
    if (Testcase == 32 || Testcase == 31) NumPlots = 5;
    std::vector<double> c((size_t)NumPlots, 0.0);
    if (NumPlots > 1) {
        const double step = T / (NumPlots - 1);
        for (int i = 1; i < NumPlots; i++) c[i] = i * step;
    }
    if (Testcase == 32) { c[1] = 8.0; c[2] = 30.0; c[3] = 300.0; c[4] = 900.0; }
    if (Testcase == 31) { c[1] = T / 12.0; c[2] = T / 6.0; c[3] = T / 4.0; c[4] = T; }
    if (Testcase == 90 || Testcase == 91 || Testcase == 86 || Testcase == 87) {
        if (NumPlots == 5 && T == 9600) { c[1] = 1200.0; c[2] = 2400.0; c[3] = 4800.0; c[4] = 9600.0; }
        if (NumPlots == 5 && T == 160) { c[1] = 20.0; c[2] = 40.0; c[3] = 80.0; c[4] = 160.0; }
    }
    if ((Testcase == 33 || Testcase == 36) && NumPlots == 7 && T == 50) {
        c[1] = 5.0; c[2] = 10.0; c[3] = 20.0; c[4] = 30.0; c[5] = 40.0; c[6] = 50.0;
    }
    return c;
}

inline void check(int rc, esdg_deviceclass* h, const char* what) {
    if (rc != ESDG_OK)
        throw std::runtime_error(std::string("esdg ") + what + " failed (" + std::to_string(rc) +
                                 "): " + esdg_last_error(h));
}

class deviceclass {
  public:
    // occa::device-like member: main.cpp:986 prints device.bytesAllocated()
    struct device_view {
        esdg_deviceclass* h = nullptr;
        double bytesAllocated() const { return (double)esdg_bytes_allocated(h); }
        void finish() const {}
    } device;
    // occa::memory-like member: main.cpp:1051 calls o_q.copyTo(q)
    struct q_view {
        esdg_deviceclass* h = nullptr;
        void copyTo(double* q) const { check(esdg_copy_q_to_host(h, q), h, "copy_q_to_host"); }
        void copyFrom(const double* q) const { check(esdg_copy_q_from_host(h, q), h, "copy_q_from_host"); }
    } o_q;

    // deviceclass(rank, argc, argv): the reference picks Serial/OpenMP/OpenCL/
    // CUDA from argv[1]; here every mode runs on the GPU, rank r on device r
    // modulo the device count chosen by the runtime (device_id = -1 keeps the
    // current device).
    deviceclass(const int rank, const int argc, char* argv[]) {
        (void)argc; (void)argv;
        check(esdg_deviceclass_create(rank, -1, &h_), nullptr, "create");
        device.h = h_;
        o_q.h = h_;
    }
    deviceclass(const deviceclass&) = delete;
    deviceclass& operator=(const deviceclass&) = delete;
    virtual ~deviceclass() {
        if (h_) esdg_deviceclass_destroy(h_);
    }

    void initDeviceVariables(const int N, const int Nelem, const int Nfaces, const int rank, const int rkSSP,
                             const int NEpad, const int NEsurfpad, const int Nedgepad, const int NAvgPad, const int ES,
                             const int Testcase, const double epsilon_0, const double sigma_max,
                             const double sigma_min, const double PosPresTOL, const double geomface,
                             const double g_const, const int PositivityPreserving, const int ArtificialViscosity,
                             const int DiscBottom, const double h_0, const int PartialDry, const int FrictionTerms,
                             const int CalcArrivalTimes, const int CreateTimeSeries, const int CalcMaximumElevation) {
        Nelem_ = Nelem;
        Nfaces_ = Nfaces;
        ngl_ = N + 1;
        h0_ = h_0;
        series_ = CreateTimeSeries;
        arrival_ = CalcArrivalTimes;
        max_elev_ = CalcMaximumElevation;
        check(esdg_init_device_variables(h_, N, Nelem, Nfaces, rank, rkSSP, NEpad, NEsurfpad, Nedgepad, NAvgPad, ES,
                                         Testcase, epsilon_0, sigma_max, sigma_min, PosPresTOL, geomface, g_const,
                                         PositivityPreserving, ArtificialViscosity, DiscBottom, h_0, PartialDry,
                                         FrictionTerms, CalcArrivalTimes, CreateTimeSeries, CalcMaximumElevation),
              h_, "initDeviceVariables");
    }

    void buildDeviceKernels(const int KernelVersion, const int KernelVersionSTD, const int Testcase,
                            const int FluxDifferencing, const int NumFlux, const int rkSSP,
                            const int ArtificialViscosity, const int PositivityPreserving, const int DiscBottom) {
        check(esdg_build_device_kernels(h_, KernelVersion, KernelVersionSTD, Testcase, FluxDifferencing, NumFlux,
                                        rkSSP, ArtificialViscosity, PositivityPreserving, DiscBottom),
              h_, "buildDeviceKernels");
    }

    void copyPartialDryData(const double* DCentralFD, const double* DforwardFD, const double* DbackwardFD) {
        check(esdg_copy_partial_dry_data(h_, DCentralFD, DforwardFD, DbackwardFD), h_, "copyPartialDryData");
    }

    // deviceclass::copyTimeSeriesIDs (src/deviceclass.cpp:556-573): global
    // node ids of the seven gauges, in this argument order
    void copyTimeSeriesIDs(const int chennai, const int paradip, const int tuticorin, const int visakhapatnam,
                           const int kochi, const int mormugao, const int okha) {
        const int ids[7] = {chennai, paradip, tuticorin, visakhapatnam, kochi, mormugao, okha};
        for (int k = 0; k < 7; ++k) gauge_id_[k] = ids[k];
    }

    void copyDeviceVariables(const int PositivityPreserving, const int Nelem, const double* GLw,
                             const double* normalsX, const double* normalsY, const double* Scal, const double* y_xi,
                             const double* y_eta, const double* x_xi, const double* x_eta, const double* b,
                             const double* Bx, const double* By, const double* Dmat, const double* Dstrong,
                             const double* Dhat, const double* J, const double* x_phy, const double* y_phy,
                             const double* q, const double* ElementSizes, const double* gRK, const double* Qt,
                             const double* VdmInv, const int* ElemEdgeMasterSlave, const int* ElemEdgeOrientation,
                             const int* ElemToEdge, const int* EdgeData, const int* EdgeReversed) {
        check(esdg_copy_device_variables(h_, PositivityPreserving, Nelem, GLw, normalsX, normalsY, Scal, y_xi, y_eta,
                                         x_xi, x_eta, b, Bx, By, Dmat, Dstrong, Dhat, J, x_phy, y_phy, q,
                                         ElementSizes, gRK, Qt, VdmInv, ElemEdgeMasterSlave, ElemEdgeOrientation,
                                         ElemToEdge, EdgeData, EdgeReversed),
              h_, "copyDeviceVariables");
    }

    // Global arrays for the outputs of DGtimeloop on rank 0
    // (deviceclass::initGlobalVars, src/deviceclass.cpp:1424-1444): b, x, y
    // and the J array main.cpp passes, copied.
    void initGlobalVars(const int Nelem_glb, const double* b, const double* x, const double* y, const double* J) {
        const size_t n = (size_t)Nelem_glb * ngl_ * ngl_;
        Nelem_global_ = Nelem_glb;
        b_.assign(b, b + n);
        x_.assign(x, x + n);
        y_.assign(y, y + n);
        J_.assign(J, J + n);
    }
    void freeGlobalVars() {
        b_.clear(); x_.clear(); y_.clear(); J_.clear();
    }

    // deviceclass::DGtimeloop (src/deviceclass.cpp:630-1335): the engine's
    // time loop, paused at the plot checkpoints, where this facade writes the
    // reference's outputs from the state at that time: the solution plot
    // (PlotVar 1 or 2), the element viscosity (artificial viscosity on and
    // PlotVar != 0; the sensor of the state at the checkpoint, where the
    // reference plots the one of the previous step's last stage), total
    // entropy and mass (EntropyPlot, through DGBasis.calcTotalEntropy /
    // calcTotalMass of the caller's basis object), the tide-gauge series
    // (CreateTimeSeries, ids from copyTimeSeriesIDs), and at the end the
    // arrival times and maximum elevation fields.  Files go to movie/, as
    // the reference's.
    template <class MPIT, class PartT, class RKT, class BasisT, class SWT>
    void DGtimeloop(const int NumElements, const int Nfaces, MPIT MPI, const PartT MeshSplit, RKT RK,
                    BasisT DGBasis, SWT SW_Problem, const double globalMinEleSize, const double CFL,
                    const double DFL, const double T, const int Testcase, const int ArtificialViscosity,
                    const int rkSSP, int NumPlots, const int NumTimeChecks, const double g_const, const int PlotVar,
                    const int EntropyPlot, const int PositivityPreserving, const int DiscBottom) {
        (void)MPI; (void)MeshSplit; (void)SW_Problem; (void)NumTimeChecks;
        const std::vector<double> cp = plot_checkpoints(NumPlots, Testcase, T);
        const bool outputs = NumPlots > 0;
        if (outputs && b_.empty())
            throw std::runtime_error("esdg DGtimeloop: plots need initGlobalVars (b, x, y, J) first");
        std::vector<double> q, ent_t, ent, mass_v, ser_t, visc;
        std::vector<double> ser[7];
        auto checkpoint = [&](int plotCount, double t, bool in_loop) {
            q.resize((size_t)NumElements * ngl_ * ngl_ * 3);
            check(esdg_copy_q_to_host(h_, q.data()), h_, "copy_q_to_host");
            tecplot::solution(NumElements, ngl_, PlotVar, x_.data(), y_.data(), q.data(), b_.data(), plotCount, h0_);
            if (in_loop && ArtificialViscosity == 1 && PlotVar != 0) {
                visc.resize((size_t)NumElements);
                check(esdg_copy_visc_to_host(h_, visc.data()), h_, "copy_visc_to_host");
                tecplot::viscosity(NumElements, ngl_, x_.data(), y_.data(), visc.data(), plotCount);
            }
            if (EntropyPlot) {
                double S = 0.0, M = 0.0;
                DGBasis.calcTotalEntropy(g_const, q.data(), b_.data(), J_.data(), &S);
                DGBasis.calcTotalMass(q.data(), J_.data(), &M);
                ent_t.resize((size_t)NumPlots); ent.resize((size_t)NumPlots); mass_v.resize((size_t)NumPlots);
                ent[plotCount] = S; mass_v[plotCount] = M; ent_t[plotCount] = t;
            }
            if (series_) {
                ser_t.resize((size_t)NumPlots);
                for (auto& v : ser) v.resize((size_t)NumPlots);
                // output columns Chennai, Tuticorin, Visakhapatnam, Paradip,
                // Kochi, Mormugao, Okha from the ids in copyTimeSeriesIDs'
                // argument order; before the loop the reference records the
                // first four only
                static const int arg_of_col[7] = {0, 2, 3, 1, 4, 5, 6};
                const int n2 = ngl_ * ngl_;
                for (int c = 0; c < (in_loop ? 7 : 4); ++c) {
                    const int gid = gauge_id_[arg_of_col[c]];
                    const long id = (long)(gid / n2) * 2 * n2 + gid;
                    ser[c][plotCount] = q[id] + b_[gid] - h0_;
                }
                ser_t[plotCount] = t;
            }
        };
        double t = 0.0;
        int steps = 0, plotCount = 0;
        if (outputs && t >= cp[0]) checkpoint(plotCount++, t, false);
        check(esdg_set_pause(h_, plotCount < NumPlots ? cp[plotCount] : INFINITY), h_, "set_pause");
        check(esdg_dg_timeloop(h_, NumElements, Nfaces, RK.rkStages, RK.CoeffsA, RK.CoeffsB, RK.CoeffsC,
                               globalMinEleSize, CFL, DFL, T, Testcase, ArtificialViscosity, rkSSP, NumPlots,
                               NumTimeChecks, g_const, PlotVar, EntropyPlot, PositivityPreserving, DiscBottom, 0, &t,
                               &steps),
              h_, "DGtimeloop");
        while (plotCount < NumPlots && t >= cp[plotCount]) {
            checkpoint(plotCount++, t, true);
            if (!(t < T)) break;
            check(esdg_set_pause(h_, plotCount < NumPlots ? cp[plotCount] : INFINITY), h_, "set_pause");
            check(esdg_resume(h_, &t, &steps), h_, "DGtimeloop (resume)");
        }
        check(esdg_set_pause(h_, INFINITY), h_, "set_pause");
        if (EntropyPlot && outputs) {
            tecplot::entropy(NumPlots, ent_t.data(), ent.data());
            tecplot::mass(NumPlots, ent_t.data(), mass_v.data());
        }
        if (series_ && outputs) tecplot::gauges(NumPlots, ser_t.data(), ser);
        if (arrival_ || max_elev_) {
            std::vector<double> v((size_t)NumElements * ngl_ * ngl_);
            if (arrival_) {
                check(esdg_copy_arrival_times(h_, v.data()), h_, "copy_arrival_times");
                tecplot::nodal("Arrivals.tec", "Arrivals.tec", "Arrivaltime", NumElements, ngl_, x_.data(), y_.data(),
                               v.data());
            }
            if (max_elev_) {
                check(esdg_copy_maximum_elevation(h_, v.data()), h_, "copy_maximum_elevation");
                tecplot::nodal("MaximumElevations.tec", "MaximumElevations.tec", "MaximumElevation", NumElements,
                               ngl_, x_.data(), y_.data(), v.data());
            }
        }
        last_t_ = t;
        last_steps_ = steps;
    }

    void freeOccaVars(const int rkSSP, const int PositivityPreserving, const int ArtificialViscosity) {
        check(esdg_free_occa_vars(h_, rkSSP, PositivityPreserving, ArtificialViscosity), h_, "freeOccaVars");
    }

    // engine extras
    // the per-node analysis outputs of src/deviceclass.cpp:1296-1309, which
    // the reference writes as Tecplot files at the end of DGtimeloop
    void copyArrivalTimes(double* out) { check(esdg_copy_arrival_times(h_, out), h_, "copyArrivalTimes"); }
    void copyMaximumElevation(double* out) {
        check(esdg_copy_maximum_elevation(h_, out), h_, "copyMaximumElevation");
    }
    esdg_deviceclass* handle() const { return h_; }
    double last_time() const { return last_t_; }
    int last_steps() const { return last_steps_; }

  private:
    esdg_deviceclass* h_ = nullptr;
    int Nelem_ = 0, Nfaces_ = 0, ngl_ = 0, Nelem_global_ = 0;
    double h0_ = 0.0;
    int series_ = 0, arrival_ = 0, max_elev_ = 0;
    int gauge_id_[7] = {0, 0, 0, 0, 0, 0, 0};
    std::vector<double> b_, x_, y_, J_;
    double last_t_ = 0.0;
    int last_steps_ = 0;
};

}  // namespace esdg_dropin
