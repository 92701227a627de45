/*
 * esdg_b200.h -- C ABI of the B200 ES-DGSEM shallow-water engine.
 *
 * The device entry points replace the OCCA-backed class `deviceclass` of
 * ESDGSEM_MPIOCCA (include/deviceclass.h:28-138, src/deviceclass.cpp) one
 * for one: same call order, same arguments (MPI/partition/basis objects are
 * passed as the plain numbers the time loop reads from them), host arrays
 * borrowed and copied, device buffers owned by the handle.  Every function
 * returns 0 on success or a negative ESDG_E* code; esdg_last_error() gives
 * the message.  Only plain C types cross this boundary.
 *
 * The set-up entry points (esdg_mesh_*, esdg_basis, ...) build the host
 * arrays that the reference's main.cpp and src/{basis,Mesh,SW2D,
 * MeshPartitioning,RungeKutta}.cpp build before calling deviceclass.
 */
#ifndef ESDG_B200_H
#define ESDG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define ESDG_OK 0
#define ESDG_E_ARG (-1)          /* bad argument or call order            */
#define ESDG_E_UNSUPPORTED (-2)  /* option outside the rebuilt hot path   */
#define ESDG_E_CUDA (-3)         /* CUDA runtime error                     */
#define ESDG_E_NONFINITE (-4)    /* solution became NaN/inf (step stopped) */
#define ESDG_E_IO (-5)           /* mesh / input file error                */
#define ESDG_E_NOMEM (-6)        /* device allocation failed               */

typedef struct esdg_deviceclass esdg_deviceclass;

/* deviceclass::deviceclass(rank, argc, argv) -- include/deviceclass.h:31,
 * src/deviceclass.cpp:20-103 (device selection).  device_id < 0 picks the
 * current CUDA device. */
int esdg_deviceclass_create(int rank, int device_id, esdg_deviceclass** out);

/* deviceclass::initDeviceVariables -- include/deviceclass.h:32-57,
 * src/deviceclass.cpp:108-345 (constants + device allocations).
 * CalcArrivalTimes / CalcMaximumElevation allocate the per-node analysis
 * outputs that every time step updates (read them with
 * esdg_copy_arrival_times / esdg_copy_maximum_elevation); h_0 is the
 * still-water level they are measured from.  CreateTimeSeries is accepted
 * and ignored. */
int esdg_init_device_variables(esdg_deviceclass* d, int N, int Nelem, int Nfaces, int rank, int rkSSP, int NEpad,
                               int NEsurfpad, int Nedgepad, int NAvgPad, int ES, int Testcase, double epsilon_0,
                               double sigma_max, double sigma_min, double PosPresTOL, double geomface,
                               double g_const, int PositivityPreserving, int ArtificialViscosity, int DiscBottom,
                               double h_0, int PartialDry, int FrictionTerms, int CalcArrivalTimes,
                               int CreateTimeSeries, int CalcMaximumElevation);

/* deviceclass::copyDeviceVariables -- include/deviceclass.h:78-107,
 * src/deviceclass.cpp:576-626.  Array sizes: K=Nelem elements, F faces,
 * n=N+1: nodal [K*n*n], q/gRK/Qt [K*3*n*n], face [F*n], matrices [n*n],
 * GLw [n], ElementSizes [K], element tables [K*4], EdgeData [F*8],
 * EdgeReversed [F]. */
int esdg_copy_device_variables(esdg_deviceclass* d, int PositivityPreserving, int Nelem, const double* GLw,
                               const double* normalsX, const double* normalsY, const double* Scal,
                               const double* y_xi, const double* y_eta, const double* x_xi, const double* x_eta,
                               const double* b, const double* Bx, const double* By, const double* Dmat,
                               const double* Dstrong, const double* Dhat, const double* J, const double* x_phy,
                               const double* y_phy, const double* q, const double* ElementSizes, const double* gRK,
                               const double* Qt, const double* VdmInv, const int* ElemEdgeMasterSlave,
                               const int* ElemEdgeOrientation, const int* ElemToEdge, const int* EdgeData,
                               const int* EdgeReversed);

/* deviceclass::copyPartialDryData -- include/deviceclass.h:69-71,
 * src/deviceclass.cpp:546-553: the finite-difference matrices [n*n] of the
 * partial-dry volume term (basis::FiniteDifferenceOperators, esdg_basis_fd).
 * Only with PartialDry = 1 at esdg_init_device_variables; required before
 * the first time step or RHS then. */
int esdg_copy_partial_dry_data(esdg_deviceclass* d, const double* DCentralFD, const double* DforwardFD,
                               const double* DbackwardFD);

/* deviceclass::buildDeviceKernels -- include/deviceclass.h:60-68,
 * src/deviceclass.cpp:349-544 (kernel selection; here: choice among the
 * compiled sm_100a instantiations). */
int esdg_build_device_kernels(esdg_deviceclass* d, int KernelVersion, int KernelVersionSTD, int Testcase,
                              int FluxDifferencing, int NumFlux, int rkSSP, int ArtificialViscosity,
                              int PositivityPreserving, int DiscBottom);

/* deviceclass::DGtimeloop -- include/deviceclass.h:113-133,
 * src/deviceclass.cpp:630-1335.  The RungeKutta object is passed as its
 * tables (rkStages, CoeffsA/B/C); globalMinEleSize as computed by
 * basis::calcElementSizes.  max_steps > 0 additionally caps the number of
 * steps (the reference loop is time-driven only).  The plot and
 * time-series arguments (NumPlots, NumTimeChecks, PlotVar, EntropyPlot) are
 * accepted and not used here: the C ABI writes no files.  The reference's
 * outputs at its plot checkpoints are written by the C++ facade
 * (include/esdg_deviceclass.hpp) around esdg_set_pause / esdg_resume below.
 * The loop stops early at a pause set with esdg_set_pause.  On return
 * *t_out / *steps_out hold the reached time and the step count. */
int esdg_dg_timeloop(esdg_deviceclass* d, int Nelem, int Nfaces, int rkStages, const double* rkA, const double* rkB,
                     const double* rkC, double globalMinEleSize, double CFL, double DFL, double T, int Testcase,
                     int ArtificialViscosity, int rkSSP, int NumPlots, int NumTimeChecks, double g_const,
                     int PlotVar, int EntropyPlot, int PositivityPreserving, int DiscBottom, int max_steps,
                     double* t_out, int* steps_out);

/* occa_device.o_q.copyTo(q) -- main.cpp:1051. */
int esdg_copy_q_to_host(esdg_deviceclass* d, double* q);
/* o_q.copyFrom(q) for restarting from a host state (src/deviceclass.cpp:593). */
int esdg_copy_q_from_host(esdg_deviceclass* d, const double* q);

/* device.bytesAllocated() -- main.cpp:986. */
long long esdg_bytes_allocated(const esdg_deviceclass* d);

/* deviceclass::freeOccaVars -- include/deviceclass.h:108-110,
 * src/deviceclass.cpp:1338-1420 (here: frees every device buffer). */
int esdg_free_occa_vars(esdg_deviceclass* d, int rkSSP, int PositivityPreserving, int ArtificialViscosity);

/* ~deviceclass. */
int esdg_deviceclass_destroy(esdg_deviceclass* d);

/* Message of the last failing call on this handle (or of the last failed
 * create when d is NULL). */
const char* esdg_last_error(const esdg_deviceclass* d);

/* One right-hand-side evaluation Qt = L(q) of the current state, as the
 * stage body of src/deviceclass.cpp:957-1094 computes it before the RK
 * update (AV terms included when enabled).  Qt_host [K*3*n*n]; visc_host
 * [K] (optional, AV only) receives the element viscosity used. */
int esdg_compute_rhs(esdg_deviceclass* d, double* Qt_host, double* visc_host);

/* Launch on the given cudaStream_t (NULL restores the handle's own stream).
 * Lets a caller order the engine's kernels with its own work and time them
 * with its own events. */
int esdg_set_stream(esdg_deviceclass* d, void* cuda_stream);

/* Checkpoints of the time loop (src/deviceclass.cpp:797-838, 1143-1147: the
 * reference writes its plots, entropy/mass and gauge series when, after a
 * step, t >= the next checkpoint; one checkpoint per step).
 * esdg_set_pause(d, t_pause): the following esdg_dg_timeloop / esdg_resume
 * stops before a step starts once t >= t_pause, provided a step ran since
 * the call began (non-finite t_pause: no pause).  Stepping is unchanged:
 * dt is clipped only at T, as in the reference.  esdg_resume(d, t, steps)
 * continues a paused loop (at least one step) until the next pause, T or the
 * step cap; on a finished loop it returns at once.  Both return
 * ESDG_E_NONFINITE / ESDG_E_CUDA as esdg_dg_timeloop does.  (No counterpart
 * call in the reference: its DGtimeloop stops at checkpoints internally.) */
int esdg_set_pause(esdg_deviceclass* d, double t_pause);
int esdg_resume(esdg_deviceclass* d, double* t_out, int* steps_out);

/* Test hook of the bounded bulk-copy waits (no counterpart in the
 * reference; for tests only).  The persistent element kernels wait on each
 * tile's bulk copies with a clock-cycle limit; a copy that never lands makes
 * the CTA record a time-out, let its other copies in flight land (bounded as
 * well) and return, and the run returns ESDG_E_CUDA.  wait_limit_cycles sets
 * that limit (0: the default, about 2 s); skip_tile >= 0 names a tile whose
 * copies are never issued, so that its wait runs out (-1: none).  Takes
 * effect for the following launches (the step graph is captured again). */
int esdg_debug_bulk_wait_test(esdg_deviceclass* d, long long wait_limit_cycles, int skip_tile);

/* Advance the resident state by up to nsteps steps (same step as
 * esdg_dg_timeloop) without any host copy of q; the device-side time and
 * step count continue from the previous call.  T is the end time. */
int esdg_advance(esdg_deviceclass* d, int nsteps, double T, double* t_out, int* steps_out);

/* Advance nsteps real steps launching kernel by kernel (no graph) with CUDA
 * events recorded on the launching stream around the face-flux and the
 * element launches; returns their average durations in ms per stage.  All
 * nsteps steps are queued before the events are read (1 <= nsteps <= 1000),
 * so the kernels run back to back as in the captured step. */
int esdg_profile_steps(esdg_deviceclass* d, int nsteps, double* face_ms, double* elem_ms);

/* Element viscosity of the last step (AV only) [K]. */
int esdg_copy_visc_to_host(esdg_deviceclass* d, double* visc);

/* The analysis outputs as DGtimeloop reads them back at its end
 * (src/deviceclass.cpp:1296-1309), per node [K*n*n]: the arrival time
 * (okl/Analysis/ArrivalTimes.okl; 1000.0 where the surface never departed
 * from h_0 by more than 5e-5) and the maximum of h + b - h_0 since the
 * start, from 0 (okl/Analysis/MaximumElevation.okl).  ESDG_E_ARG unless
 * enabled at esdg_init_device_variables. */
int esdg_copy_arrival_times(esdg_deviceclass* d, double* arrival_times);
int esdg_copy_maximum_elevation(esdg_deviceclass* d, double* maximum_elevation);

/* Number of kernel launches issued by the engine since creation (graph
 * replays count the kernels inside the graph). */
long long esdg_kernel_launches(const esdg_deviceclass* d);

/* Same evaluation as esdg_compute_rhs, for callers that must not allocate
 * device memory (no counterpart in the reference): hosts whose device memory
 * belongs to their own pool allocator, and serving loops that cannot afford
 * the device-wide synchronisation of cudaMalloc/cudaFree.  Every pointer is a
 * device pointer the caller owns, in the layouts of esdg_copy_device_variables
 * (Jinv = 1/J, Dmat the flux-differencing matrix); Qt [K*3*(N+1)^2] receives
 * L(q).  The scratch (packed tables, bathymetry traces, face fluxes, one step
 * state) is a fixed 16 MiB device array inside this library (2^21 doubles),
 * held by every GPU that loads it until the process exits.  A mesh needs
 * 2*F + 8*K + 5*F*(N+1) doubles of it plus the step state and an error
 * count, each table rounded up to 256 bytes; a mesh needing more than the
 * array is rejected with ESDG_E_ARG.  The first call on a device looks the
 * array's address up (cudaGetSymbolAddress) with that device current: make
 * that first call before any stream capture.  A stream given must belong to
 * the current device (ESDG_E_ARG otherwise).  All calls share the one array,
 * so calls that overlap on the GPU race; every call rewrites the parts it
 * reads.  Out-of-range connectivity is replaced by safe entries and reported
 * as ESDG_E_ARG.  Runs on `stream` (NULL: legacy default stream); the call
 * copies the count of bad connectivity entries back to the host and
 * synchronises `stream` before it returns.  The message of a failure is
 * esdg_last_error(NULL). */
int esdg_compute_rhs_noalloc(int N, int K, int F, int NumFlux, int ES, double g_const, double PosPresTOL,
                             const double* q, const double* Jinv, const double* y_xi, const double* y_eta,
                             const double* x_xi, const double* x_eta, const double* Bx, const double* By,
                             const double* b, const double* Dmat, const double* nx, const double* ny,
                             const double* scal, const int* EdgeData, const int* ElemToEdge,
                             const int* ElemEdgeMasterSlave, const int* ElemEdgeOrientation, double* Qt,
                             void* stream);

/* Element-kernel variant chosen by the engine's autotuner (no counterpart
 * in the reference): before the first step graph is captured the engine
 * times each compiled variant of the element kernel on the mesh (in the
 * step's own update mode, on copies of q and gRK, each launch after an
 * L2-sized flush) and keeps the fastest.  Variants 0-2: one thread per node
 * (CTAs per SM the register budget is cut for, 2 or 3; bulk-copy pipeline
 * depth, 2 or 3 tiles); variants 3-4 (N = 2..5): one thread per element row
 * and column, each symmetric two-point flux evaluated once (two tile sizes).
 * *ctas_per_sm and *stages receive the choice (0: the one-shot kernel is
 * used), ms_variants3 [3] (may be NULL) the measured launch times of
 * variants 0-2 (esdg_element_variants reports all of them).
 * ESDG_E_ARG before the tuning ran. */
int esdg_tuned_config(const esdg_deviceclass* d, int* ctas_per_sm, int* stages, float* ms_variants3);

/* All element-kernel variants (no counterpart in the reference): *count
 * the number compiled, *chosen the one the steps use (-1: the one-shot
 * kernel), and for the first cap of them ms [cap] the autotuner's launch
 * times (0: not timed) and ctas_per_sm [cap] the resident CTAs per SM
 * (0: not available for this degree / element count).  Pointers may be
 * NULL.  ESDG_E_ARG before the tuning ran (or a variant was fixed). */
int esdg_element_variants(const esdg_deviceclass* d, int* chosen, int* count, float* ms, int* ctas_per_sm,
                          int cap);

/* Fixes the element-kernel variant for every later step and RHS (no
 * counterpart in the reference); -1 returns to the autotuner's choice.
 * Call after buildDeviceKernels; re-captures the step graph if there is one.
 * ESDG_E_UNSUPPORTED for a variant that is not available here.  All
 * variants compute the same bits. */
int esdg_set_element_variant(esdg_deviceclass* d, int variant);

/* Device addresses of the solution q [K][3][(N+1)^2], the bathymetry b
 * [K][(N+1)^2] and VdmInv [(N+1)^2] owned by the engine (no counterpart in
 * the reference), for device-side consumers such as the indicator's
 * training-data extraction.  Valid until esdg_free_occa_vars. */
int esdg_state_pointers(esdg_deviceclass* d, const double** q, const double** b, const double** VdmInv);

/* Troubled-cell indicator of the artificial-viscosity path (no counterpart
 * in the reference; call after esdg_build_device_kernels with
 * ArtificialViscosity=1):
 *   mode 0  the reference's path: the modal sensor
 *           (okl/ShockCapturing/ShockCapturing.okl:17-234) and the viscous
 *           terms on every element (the default);
 *   mode 1  the modal sensor with the active set: the BR1 gradient and the
 *           viscous terms run only on elements with viscosity > 0 and their
 *           face neighbours (everywhere else they are exactly zero), so the
 *           solution is the same as with mode 0;
 *   mode 2  the learned indicator with the active set: the network whose
 *           FP32 parameter block (esdg_mlp_layout(N+1).total floats) is
 *           `params` sets viscosity 0 where it predicts
 *           sigma < sigma_min - margin and eps0 where it predicts
 *           sigma > sigma_max + margin; the modal sensor decides every other
 *           element (the ramp band, positivity check failures, modal energy
 *           near ZeroTOL).  N in 3..5.  At N = 3 features, network and
 *           sensor fallback run as one fused pass over the state;
 *   mode 3  mode 2's decisions computed by three separate passes (feature
 *           rows, batched network, sensor) at every degree; the same
 *           numbers as mode 2.
 * params/nparams/margin are ignored for modes 0 and 1. */
int esdg_set_indicator(esdg_deviceclass* d, int mode, const float* params, int nparams, float margin);

/* Schedule of the learned indicator (modes 2 and 3; no counterpart in the
 * reference): every_stage != 0 (the default) evaluates it at every RK stage,
 * as the reference evaluates its sensor (src/deviceclass.cpp:1043-1046);
 * 0 evaluates it once per step, at the step start, and keeps the
 * viscosity and the active set for the step's stages -- one more
 * approximation of the learned path, whose deviation from the plain path is
 * measured like the network's.  Modes 0 and 1 are exact and always run
 * every stage.  Re-captures the step graph. */
int esdg_set_indicator_every_stage(esdg_deviceclass* d, int every_stage);

/* Decision counts accumulated over indicator launches: [0] elements the
 * network set to zero, [1] set to eps0, [2] decided by the modal sensor,
 * [3] elements with nonzero viscosity; reset != 0 zeroes them. */
int esdg_indicator_stats(esdg_deviceclass* d, unsigned long long* counts4, int reset);

/* ------------------------------------------------------------------------
 * Batched ensemble (no counterpart in the reference, which runs one mesh
 * per process): independent instances of one polynomial degree N advanced
 * together, each kernel launch covering every instance, each instance with
 * its own time, time step, end time and step cap.  Instances are added and
 * removed between advances; the captured step graph stays valid.
 * ---------------------------------------------------------------------- */

typedef struct esdg_ensemble esdg_ensemble;

/* Capacity for max_instances instances holding up to K_capacity elements
 * and F_capacity faces in total; the solver switches are those of
 * initDeviceVariables/buildDeviceKernels, shared by every instance. */
int esdg_ensemble_create(int device_id, int N, int max_instances, int K_capacity, int F_capacity, int NumFlux, int ES,
                         double g_const, double PosPresTOL, int ArtificialViscosity, double epsilon_0,
                         double sigma_max, double sigma_min, int PositivityPreserving, int rkOrder, int rkSSP,
                         esdg_ensemble** out);

/* Adds one instance (host arrays as for esdg_copy_device_variables, its own
 * numbering; J is 1/J), running until t >= T or max_steps steps (0: no cap);
 * *id receives its slot.  ESDG_E_NOMEM when no contiguous capacity is free. */
int esdg_ensemble_add(esdg_ensemble* en, int Nelem, int Nfaces, const double* normalsX, const double* normalsY,
                      const double* Scal, const double* y_xi, const double* y_eta, const double* x_xi,
                      const double* x_eta, const double* b, const double* Bx, const double* By, const double* J,
                      const double* q, const double* ElementSizes, const int* ElemEdgeMasterSlave,
                      const int* ElemEdgeOrientation, const int* ElemToEdge, const int* EdgeData, double T,
                      int max_steps, double minEleSize, double CFL, double DFL, int* id);

/* Releases an instance's slot and capacity (its results are gone). */
int esdg_ensemble_remove(esdg_ensemble* en, int id);

/* Replays the step graph nsteps times (finished instances are skipped on
 * the device) and refreshes the host copy of every instance's status. */
int esdg_ensemble_advance(esdg_ensemble* en, int nsteps);

/* The two halves of esdg_ensemble_advance: replay the step graph nsteps
 * times on the ensemble's stream without waiting, and wait for it and
 * refresh the host status -- so that several ensembles (one per degree) run
 * concurrently. */
int esdg_ensemble_launch(esdg_ensemble* en, int nsteps);
int esdg_ensemble_sync(esdg_ensemble* en);

/* Status from the last advance: time, steps taken, done flag, status
 * (0 ok, 1 non-finite wave speed). */
int esdg_ensemble_status(esdg_ensemble* en, int id, double* t, int* steps, int* done, int* status);

/* Copies an instance's q [Nelem*3*(N+1)^2] to the host. */
int esdg_ensemble_copy_q(esdg_ensemble* en, int id, double* q);

/* Largest free contiguous element and face ranges and the free slot count. */
int esdg_ensemble_free_capacity(const esdg_ensemble* en, int* K_largest, int* F_largest, int* free_slots);

long long esdg_ensemble_bytes(const esdg_ensemble* en);
long long esdg_ensemble_kernel_launches(const esdg_ensemble* en);

/* Runs on the caller's stream (NULL: the ensemble's own); re-captures the
 * step graph. */
int esdg_ensemble_set_stream(esdg_ensemble* en, void* cuda_stream);
/* esdg_set_indicator / esdg_indicator_stats for every instance of the
 * ensemble (re-captures the step graph). */
int esdg_ensemble_set_indicator(esdg_ensemble* en, int mode, const float* params, int nparams, float margin);
int esdg_ensemble_indicator_stats(esdg_ensemble* en, unsigned long long* counts4, int reset);
/* esdg_set_indicator_every_stage for every instance of the ensemble. */
int esdg_ensemble_set_indicator_every_stage(esdg_ensemble* en, int every_stage);
/* esdg_set_element_variant / esdg_element_variants for the ensemble's
 * element kernel (no counterpart in the reference). */
int esdg_ensemble_set_element_variant(esdg_ensemble* en, int variant);
int esdg_ensemble_element_variants(const esdg_ensemble* en, int* chosen, int* count, float* ms, int* ctas_per_sm,
                                   int cap);
const char* esdg_ensemble_last_error(const esdg_ensemble* en);
int esdg_ensemble_destroy(esdg_ensemble* en);

/* ------------------------------------------------------------------------
 * Learned troubled-cell indicator: training kernels (no counterpart in the
 * reference).  A 3-layer MLP (F -> 32 -> 32 -> 1, ReLU) predicting the modal
 * shock sensor's sigma = log10(energy ratio) of an element
 * (okl/ShockCapturing/ShockCapturing.okl:131-204) from its features; BF16
 * weights and activations on the tensor cores, FP32 accumulation, FP32
 * master weights.  ngl = N+1 in 3..6.  Every pointer is a device pointer;
 * calls are asynchronous on `stream` (NULL: legacy default stream).
 * Failures are described by esdg_last_error(NULL).
 * ---------------------------------------------------------------------- */

/* Parameter block layout in floats: kp (row length of X and W1), offsets
 * of W1[32][kp], b1[32], W2[32][32], b2[32], w3[32], b3, and the total. */
int esdg_mlp_layout(int ngl, int* out8);

/* Feature rows X [K][kp] (bf16) of the elements of q/b; when tgt is given,
 * the training target clamp(sigma, -12, 0) - s_eta [K] (float); when seta
 * is given, s_eta [K] (the log energy fraction of h + b's deviation). */
int esdg_mlp_features(int ngl, int K, const double* q, const double* b, const double* VdmInv, double ZeroTOL, void* X,
                      float* tgt, float* seta, void* stream);

/* Pb (bf16) = P (float) over the whole block. */
int esdg_mlp_cast(int ngl, const float* P, void* Pb, void* stream);

/* y [M] = network output for the rows of X; `blocks` CTAs of 4 warps. */
int esdg_mlp_forward(int ngl, int M, const void* X, const float* P, const void* Pb, float* y, int blocks,
                     void* stream);

/* Per-warp partial gradients of (1/M) sum (y - t)^2: partial [blocks*4][total]
 * (slot b3+1 of each row: that warp's sum of squared errors). */
int esdg_mlp_backward(int ngl, int M, const void* X, const float* tgt, const float* P, const void* Pb,
                      float* partial, int blocks, void* stream);

/* G = sum of the `rows` partial rows (fixed order), then one Adam step
 * (step >= 1) on P, m, v, refreshing Pb. */
int esdg_mlp_adam(int ngl, int rows, const float* partial, float* G, float* P, void* Pb, float* m, float* v,
                  float lr, float beta1, float beta2, float eps, int step, void* stream);

/* ------------------------------------------------------------------------
 * Host set-up (no GPU needed).
 * ---------------------------------------------------------------------- */

typedef struct esdg_mesh esdg_mesh;

/* basis::basis (src/basis.cpp:28-188): LGL nodes/weights [n], Gauss
 * nodes/weights [n], D (flux-differencing form when FluxDifferencing),
 * D0 (plain collocation derivative), Dstrong, Dhat, VdmInv [n*n]. */
int esdg_basis(int N, int FluxDifferencing, double* xGL, double* wGL, double* xG, double* wG, double* D, double* D0,
               double* Dstrong, double* Dhat, double* VdmInv);

/* basis::FiniteDifferenceOperators (src/basis.cpp:190-229): the central,
 * forward and backward two-point difference matrices [n*n] on the LGL
 * nodes used by the partial-dry volume term. */
int esdg_basis_fd(int N, double* DCentralFD, double* DforwardFD, double* DbackwardFD);

/* Mesh::GenerateMesh (src/Mesh.cpp:316-696) for a Cartesian grid.
 * periodic_rows / periodic_cols are the reference's PeriodicBD_X /
 * PeriodicBD_Y (wrap of the horizontal / vertical faces). */
int esdg_mesh_cartesian(int N, double xL, double xR, double yL, double yR, int NX, int NY, int periodic_rows,
                        int periodic_cols, esdg_mesh** out);

/* Structured curved grid x -> x + amp*Lx*sin(2pi(x-xL)/Lx)sin(2pi(y-yL)/Ly)
 * (y likewise) with every side given as an order-m boundary curve, i.e. the
 * ISM-V2 mesh that esdg_mesh_write_ism2 writes; rotate_seed != 0 rotates
 * element corner numbering pseudo-randomly (faces of all orientations). */
int esdg_mesh_mapped(int N, double xL, double xR, double yL, double yR, int NX, int NY, double amp, int m,
                     unsigned rotate_seed, esdg_mesh** out);

/* Mesh::ReadMesh (src/Mesh.cpp:698-1503): ISM-V2 reader. */
int esdg_mesh_read_ism2(int N, const char* path, int read_bottom, int convert_km, esdg_mesh** out);
int esdg_mesh_write_ism2(const esdg_mesh* m, const char* path);

/* Curvilinear geometry on the device (the set-up's geometry of
 * src/Mesh.cpp:1000-1081, 1619-1650, 1667-1808 -- boundary-curve transfinite
 * map, collocation metric terms, Jacobian, side normals -- with every
 * operation in the host set-up's order, so the same bits).  Inputs are
 * device arrays: per element its 4 corners (x, y) [K][4][2], per side a
 * curve flag [K][4] and curve_order + 1 Chebyshev-Gauss-Lobatto samples
 * (x, y) [K][4][curve_order+1][2] (sides 0 bottom, 1 right, 2 top, 3 left,
 * as in an ISM-V2 file); outputs x, y, x_xi, x_eta, y_xi, y_eta and J
 * (not 1/J) [K][N+1][N+1], and the outward unit normal and scale factor of
 * each side node nx_side, ny_side, scal_side [K][4][N+1].  Runs on `stream`
 * (NULL: the legacy default stream) without synchronising; allocates
 * nothing.  esdg_mesh_element_curves exports a host mesh's corners, flags
 * and samples in that layout (all arrays NULL: only *curve_order). */
int esdg_mesh_element_curves(const esdg_mesh* m, int* curve_order, double* corners, int* curved, double* curves);
int esdg_geometry_device(int N, int K, int curve_order, const double* corners, const int* curved,
                         const double* curves, double* x, double* y, double* x_xi, double* x_eta, double* y_xi,
                         double* y_eta, double* J, double* nx_side, double* ny_side, double* scal_side, void* stream);

/* Sea-surface uplift of a rectangular fault on the device (Okada 1985
 * vertical displacement of strike-slip and dip-slip dislocations,
 * src/okada.cpp:33-249), one value per node: out[i] = uplift, or
 * out[i] += uplift with add != 0.  fault = {x0, y0, depth, length, width,
 * strike, rake, dip, slip} (angles in degrees).  mercator != 0: the
 * reference's geometry -- x, y in Mercator kilometres, (x0, y0) the
 * epicentre's longitude and latitude, the uplift in kilometres inside the
 * reference's box; mercator = 0: plane coordinates in metres, (x0, y0) the
 * fault centroid, the uplift in metres inside a box of half-size
 * 1.5 max(length, width) (non-finite corner terms give 0).  x, y, out are
 * device arrays of n values; runs on `stream` without synchronising and
 * allocates nothing. */
int esdg_okada_uplift(long long n, const double* x, const double* y, const double* fault, int mercator, int add,
                      double* out, void* stream);

/* Element and face counts. */
int esdg_mesh_sizes(const esdg_mesh* m, int* K, int* F);

/* Arrays as main.cpp:650-716 hands them to copyDeviceVariables (J is 1/J).
 * Any pointer may be NULL. */
int esdg_mesh_pack(const esdg_mesh* m, double* x, double* y, double* x_xi, double* x_eta, double* y_xi,
                   double* y_eta, double* Jinv, double* nx, double* ny, double* scal, double* b, int* EdgeData,
                   int* EdgeReversed, int* ElemToEdge, int* ElemEdgeMasterSlave, int* ElemEdgeOrientation);
void esdg_mesh_free(esdg_mesh* m);

/* SW2D::CalcBDerivatives (src/SW2D.cpp:1048-1105), Jinv = 1/J. */
int esdg_bottom_derivatives(int K, int N, const double* D0, const double* b, const double* y_eta, const double* y_xi,
                            const double* x_eta, const double* x_xi, const double* Jinv, double* Bx, double* By);

/* basis::calcElementSizes (src/basis.cpp:939-966); returns sqrt(min area)
 * in *minEleSize. */
int esdg_element_sizes(int K, int N, const double* wGL, const double* Jinv, double* EleSizes, double* minEleSize);

/* RungeKutta::RungeKutta (src/RungeKutta.cpp:18-90); A/B/C hold >= 5. */
int esdg_rk_coefficients(int order, int ssp, double* A, double* B, double* C, int* stages);

/* basis::L2Norm / LinfNorm / calcTotalMass / calcTotalEntropy
 * (src/basis.cpp:874-1111); qref may be NULL (then L2/Linf are skipped). */
int esdg_diagnostics(int K, int N, const double* wGL, const double* Jinv, const double* q, const double* qref,
                     const double* b, double g, double* L2, double* Linf, double* mass, double* entropy);

#ifdef __cplusplus
}
#endif

#endif /* ESDG_B200_H */
