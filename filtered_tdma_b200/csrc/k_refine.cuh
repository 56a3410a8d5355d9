// FP64 residual and convergence bookkeeping of mixed-precision iterative
// refinement (FP32 storage, FP32 inner solves, FP64 residual and solution).
//
// For one batch, with T the tridiagonal matrix of each system (A, B, C stored in
// FP32 and widened exactly to FP64) and x the current FP64 solution:
//
//     r = D - T x                      (FP64 arithmetic, stored as FP32: the
//                                       correction solve needs ~7 digits of it)
//     eta = max|r| / (max_j(|a_j| + |b_j| + |c_j|) * max|x| + max|D|)
//
// eta is the normwise backward error of x; a system has converged once
// eta <= eta_tol, and its forward error is then at most cond(T) * eta.  The
// non-periodic solvers ignore a_0 and c_{n-1} (so does this residual); periodic
// systems couple row 0 with row n-1.
#pragma once

#include "btdma_common.cuh"

namespace btdma {

constexpr unsigned char REFINE_OPEN = 0xff;      // not converged yet
constexpr unsigned char REFINE_FALLBACK = 0xfe;  // not converged after the last sweep

// One thread per system; consecutive threads read consecutive systems of a
// row (coalesced).  `sweep` = corrections applied so far.  Systems that meet
// the bound for the first time record `sweep` in iters[]; systems still open
// after this check add to *open_count.  At the last sweep open systems are
// marked REFINE_FALLBACK instead.  gate (optional): nothing to do while
// *gate == 0 (every system converged earlier).
__global__ void __launch_bounds__(256)
refine_residual_kernel(const float* __restrict__ A, const float* __restrict__ B,
                       const float* __restrict__ C, const float* __restrict__ D,
                       const double* __restrict__ X, float* __restrict__ R, int n_sys, int n_row,
                       int cyclic, int sweep, int last, double eta_tol,
                       unsigned char* __restrict__ iters, const unsigned* gate,
                       unsigned* open_count) {
    if (gate != nullptr && *static_cast<const volatile unsigned*>(gate) == 0u) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_sys) return;
    const size_t ns = (size_t)n_sys;
    const int n = n_row;
    double rmax = 0.0, xmax = 0.0, dmax = 0.0, tmax = 0.0;
    double xm = cyclic ? X[(size_t)(n - 1) * ns + i] : 0.0;  // x_{j-1}
    double x0 = X[i];
    double xc = x0;
#pragma unroll 4
    for (int j = 0; j < n; ++j) {
        const size_t o = (size_t)j * ns + i;
        double xp;  // x_{j+1}
        if (j + 1 < n)
            xp = X[o + ns];
        else
            xp = cyclic ? x0 : 0.0;
        double a = (double)A[o], c = (double)C[o];
        if (!cyclic) {
            if (j == 0) a = 0.0;
            if (j == n - 1) c = 0.0;
        }
        const double b = (double)B[o], d = (double)D[o];
        const double r = d - a * xm - b * xc - c * xp;
        R[o] = (float)r;
        rmax = fmax(rmax, fabs(r));
        xmax = fmax(xmax, fabs(xc));
        dmax = fmax(dmax, fabs(d));
        tmax = fmax(tmax, fabs(a) + fabs(b) + fabs(c));
        xm = xc;
        xc = xp;
    }
    const double scale = tmax * xmax + dmax;
    const bool ok = rmax <= eta_tol * scale;  // NaN compares false: stays open
    unsigned char it = sweep == 0 ? REFINE_OPEN : iters[i];
    if (it == REFINE_OPEN) {
        if (ok)
            it = (unsigned char)sweep;
        else if (last)
            it = REFINE_FALLBACK;
    }
    iters[i] = it;
    // one atomic per warp: the count of open systems among its lanes
    const unsigned act = __activemask();
    const unsigned open = __ballot_sync(act, it == REFINE_OPEN || it == REFINE_FALLBACK);
    if (open != 0u && (int)(threadIdx.x & 31) == __ffs(act) - 1)
        atomicAdd(open_count, (unsigned)__popc(open));
}

}  // namespace btdma
