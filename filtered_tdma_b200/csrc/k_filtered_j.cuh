// Filtered TDMA bookkeeping kernels: spectral bounds (rho) and truncation depth J.
//
// The reference keeps rho per row on the device (d_A_rho/d_C_rho, filled by
// k_set_rho from system 0's column, libs/filtered_tdma/gpu/filtered_tdma_kernels.cuh:
// 46-67) and computes J in a single 256-thread block (k_cal_J_rhs_bound, :220-261).
// Here one bound per row (max of the two) is kept, and J is computed per segment
// by a grid-wide max reduction (many blocks + atomicMax on the bit patterns of
// non-negative doubles) followed by a one-warp finalize that also resets the
// accumulators, so consecutive solves (and graph replays) need no memset.
#pragma once

#include "btdma_common.cuh"

namespace btdma {

constexpr int JRED_BLOCK = 256;

// rho_row[k] = max(|A_k/B_k|, |C_k/B_k|) of system 0 (0 where B_k == 0).
__global__ void rho_sys0_kernel(const double* __restrict__ A, const double* __restrict__ B,
                                const double* __restrict__ C, int n_sys, int n_row,
                                double* __restrict__ rho_row) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_row) return;
    const size_t off = (size_t)k * n_sys;
    const double b = B[off];
    double v = 0.0;
    if (b != 0.0) v = fmax(fabs(A[off] / b), fabs(C[off] / b));
    rho_row[k] = v;
}

// rho_row[k] = max over all systems (rho_bits zeroed by the caller).
__global__ void rho_all_kernel(const double* __restrict__ A, const double* __restrict__ B,
                               const double* __restrict__ C, int n_sys,
                               unsigned long long* __restrict__ rho_bits) {
    const int k = blockIdx.y;
    const size_t off = (size_t)k * n_sys;
    double v = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_sys; i += gridDim.x * blockDim.x) {
        const double b = B[off + i];
        if (b != 0.0) v = fmax(v, fmax(fabs(A[off + i] / b), fabs(C[off + i] / b)));
    }
    unsigned long long bits = __double_as_longlong(v);
    for (int o = 16; o > 0; o >>= 1) bits = max(bits, __shfl_xor_sync(0xffffffffu, bits, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&rho_bits[k], bits);
}

// max |D| over the first and last rows of segment blockIdx.y (or over all its
// rows when `all_rows`), accumulated into work[2*segment].
__global__ void __launch_bounds__(JRED_BLOCK)
jmax_kernel(const double* __restrict__ D, int n_sys, int n_row, int P, int all_rows,
            unsigned long long* __restrict__ work) {
    const int k = blockIdx.y;
    int r0, m;
    seg_range(n_row, P, k, r0, m);
    double v = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_sys; i += gridDim.x * blockDim.x) {
        if (all_rows) {
            for (int j = 0; j < m; ++j) v = fmax(v, fabs(D[(size_t)(r0 + j) * n_sys + i]));
        } else {
            v = fmax(v, fabs(D[(size_t)r0 * n_sys + i]));
            v = fmax(v, fabs(D[(size_t)(r0 + m - 1) * n_sys + i]));
        }
    }
    unsigned long long bits = __double_as_longlong(v);
    for (int o = 16; o > 0; o >>= 1) bits = max(bits, __shfl_xor_sync(0xffffffffu, bits, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&work[2 * k], bits);
}

// J per segment from the accumulated maxima; resets the accumulators.
//   rho   = max of rho_row over the segment's rows 1..m-1
//           (filtered_tdma.cpp:66-71, filtered_tdma_kernels.cuh:231-233);
//   eps   = eps_constant / (m*P)^2 (filtered_tdma.cpp:49-51);
//   v2 / device v1: B = q(2+q)/((1-q)(1-2rho)) * max_b (filtered_tdma_kernels.cuh:249-257),
//   host v1:        B = (max|x0| + max|xN|) q/(1-q)    (filtered_tdma.cpp:110-114),
//   J = int(log(eps/B)/log q) + 1 clamped to [0, m-1]; rho in {0} u [0.5, inf) -> m-1.
// exact (optional): set to 1 when some segment has rho >= 0.5 (the bound does
// not hold) or J >= m - 2 (the truncation keeps every row, so only the 2x2
// interface approximation would remain), else 0: the solve then takes the exact
// reduced system instead of the Filtered interface.  One warp.
__global__ void jfinal_kernel(unsigned long long* __restrict__ work, int* __restrict__ J,
                              const double* __restrict__ rho_row, int n_row, int P,
                              double eps_constant, int version, int host_semantics,
                              unsigned* __restrict__ exact) {
    bool need_exact = false;
    for (int k = threadIdx.x; k < P; k += blockDim.x) {
        int r0, m;
        seg_range(n_row, P, k, r0, m);
        double rho = 0.0;
        for (int j = 1; j < m; ++j) rho = fmax(rho, rho_row[r0 + j]);
        const double m0 = __longlong_as_double((long long)work[2 * k]);
        const double mn = __longlong_as_double((long long)work[2 * k + 1]);
        int Jk;
        if (rho == 0.0 || rho >= 0.5) {
            Jk = m - 1;
        } else {
            const double N = (double)(m * P);
            const double eps = eps_constant / (N * N);
            const double lambda_p = (1.0 + sqrt(1.0 - 4.0 * rho * rho)) * 0.5;
            const double q = rho / lambda_p;
            double bound;
            if (version == 1 && host_semantics)
                bound = (m0 + mn) * q / (1.0 - q);
            else
                bound = q * (2.0 + q) / ((1.0 - q) * (1.0 - 2.0 * rho)) * fmax(m0, mn);
            const double t = log(eps / bound) / log(q);
            // the float->int cast of the reference, made total for inf/NaN
            long long ti = isnan(t) ? 0 : (t >= 2147483647.0 ? 2147483647LL
                                       : (t <= -2147483648.0 ? -2147483648LL : (long long)t));
            long long Jl = ti + 1;
            if (Jl > m - 1) Jl = m - 1;
            if (Jl < 0) Jl = 0;
            Jk = (int)Jl;
        }
        J[k] = Jk;
        need_exact |= rho >= 0.5 || Jk >= m - 2;
        work[2 * k] = 0ull;
        work[2 * k + 1] = 0ull;
    }
    const bool any = __any_sync(0xffffffffu, need_exact);
    if (exact != nullptr && threadIdx.x == 0) *exact = any ? 1u : 0u;
}

}  // namespace btdma
