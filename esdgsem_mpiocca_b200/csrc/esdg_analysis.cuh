// Analysis outputs of the time loop: tsunami arrival times and the maximum
// free-surface elevation per node.
#pragma once

#include "esdg_kernels.cuh"

namespace esdg {

// Arrival times start at the sentinel 1000.0 (src/deviceclass.cpp:324-333).
__global__ void k_fill_f64(double* p, long n, double v) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) p[k] = v;
}

// After each time step, with the new time t (called after t += dt at
// src/deviceclass.cpp:1130-1141), per node:
//  * okl/Analysis/ArrivalTimes.okl:16-62: while the entry is still 1000.0,
//    record t once the free surface h + b departs from h_zero by more than
//    5e-5;
//  * okl/Analysis/MaximumElevation.okl:16-55: the running maximum of
//    h + b - h_zero, starting from 0 (src/deviceclass.cpp:337-341), taken
//    as std::max(old, new) takes it.
// Either output may be null.  One thread per node; a finished run (done
// flag) leaves both unchanged, as the reference runs no further step.
template <int N2>
__global__ void __launch_bounds__(256) k_analysis(long nodes, const double* __restrict__ q,
                                                  const double* __restrict__ B, const DevState* __restrict__ st,
                                                  double h_zero, double* __restrict__ arrival,
                                                  double* __restrict__ max_elev) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nodes || st[0].done) return;
    const long e = k / N2;
    const long nd = k - e * N2;
    const double h = q[e * 3 * N2 + nd];
    const double b = B[k];
    if (arrival && arrival[k] == 1000.0 && fabs((h + b) - h_zero) > 0.00005) arrival[k] = st[0].t;
    if (max_elev) {
        const double fs = h + b - h_zero;
        const double m = max_elev[k];
        max_elev[k] = (m < fs) ? fs : m;
    }
}

}  // namespace esdg
