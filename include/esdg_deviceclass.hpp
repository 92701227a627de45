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

#include <stdexcept>
#include <string>

#include "esdg_b200.h"

namespace esdg_dropin {

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

    void copyTimeSeriesIDs(const int, const int, const int, const int, const int, const int, const int) {}

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

    // Global arrays for plotting on rank 0 (no plots are written here).
    void initGlobalVars(const int, const double*, const double*, const double*, const double*) {}
    void freeGlobalVars() {}

    template <class MPIT, class PartT, class RKT, class BasisT, class SWT>
    void DGtimeloop(const int NumElements, const int Nfaces, MPIT MPI, const PartT MeshSplit, RKT RK,
                    BasisT DGBasis, SWT SW_Problem, const double globalMinEleSize, const double CFL,
                    const double DFL, const double T, const int Testcase, const int ArtificialViscosity,
                    const int rkSSP, int NumPlots, const int NumTimeChecks, const double g_const, const int PlotVar,
                    const int EntropyPlot, const int PositivityPreserving, const int DiscBottom) {
        (void)MPI; (void)MeshSplit; (void)DGBasis; (void)SW_Problem;
        double t = 0.0;
        int steps = 0;
        check(esdg_dg_timeloop(h_, NumElements, Nfaces, RK.rkStages, RK.CoeffsA, RK.CoeffsB, RK.CoeffsC,
                               globalMinEleSize, CFL, DFL, T, Testcase, ArtificialViscosity, rkSSP, NumPlots,
                               NumTimeChecks, g_const, PlotVar, EntropyPlot, PositivityPreserving, DiscBottom, 0, &t,
                               &steps),
              h_, "DGtimeloop");
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
    int Nelem_ = 0, Nfaces_ = 0;
    double last_t_ = 0.0;
    int last_steps_ = 0;
};

}  // namespace esdg_dropin
