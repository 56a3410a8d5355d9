// Serial Thomas kernels (P = 1): one thread per system, row-interleaved layout.
//
// Bit-identical to the reference's CPU tdma_many / tdma_cyclic_many
// (libs/pascal_tdma/cpu/tdma_local.cpp:6-52, 108-208): the same operation order,
// IEEE round-to-nearest for every operation, no fused multiply-add (the
// reference's CPU build does not contract).  The reference's own GPU kernel
// divides row 0 by B instead of multiplying by 1/B
// (libs/pascal_tdma/gpu/tdma_local_cuda.cu:43-44), so it is not the bit oracle.
//
// The forward sweep keeps the running (c', d') in registers and spills c' to the
// handle's scratch and d' to X; the backward sweep reads them back.  Loads are
// issued a block of UNR rows ahead of the arithmetic (X may alias D, so the
// compiler cannot hoist them itself).
#pragma once

#include "btdma_common.cuh"

namespace btdma {

constexpr int THOMAS_BLOCK = 128;
constexpr int THOMAS_UNR = 4;

__global__ void __launch_bounds__(THOMAS_BLOCK)
thomas_f64_kernel(const double* __restrict__ A, const double* __restrict__ B,
                  const double* __restrict__ C, const double* D, double* X,
                  double* __restrict__ Cs, int n_sys, int n_row, unsigned* status) {
    using E = Exact64;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_sys) return;
    const size_t ns = (size_t)n_sys;

    double inv_b = E::rcp(B[i]);
    double d = E::mul(D[i], inv_b);
    double c = E::mul(C[i], inv_b);
    Cs[i] = c;
    X[i] = d;

    int j = 1;
    for (; j + THOMAS_UNR <= n_row; j += THOMAS_UNR) {
        double a[THOMAS_UNR], b[THOMAS_UNR], cc[THOMAS_UNR], dd[THOMAS_UNR];
#pragma unroll
        for (int u = 0; u < THOMAS_UNR; ++u) {
            size_t off = (size_t)(j + u) * ns + i;
            a[u] = A[off];
            b[u] = B[off];
            cc[u] = C[off];
            dd[u] = D[off];
        }
#pragma unroll
        for (int u = 0; u < THOMAS_UNR; ++u) {
            size_t off = (size_t)(j + u) * ns + i;
            double r = E::rcp(E::sub(b[u], E::mul(a[u], c)));
            d = E::mul(r, E::sub(dd[u], E::mul(a[u], d)));
            c = E::mul(r, cc[u]);
            Cs[off] = c;
            X[off] = d;
        }
    }
    for (; j < n_row; ++j) {
        size_t off = (size_t)j * ns + i;
        double a = A[off];
        double r = E::rcp(E::sub(B[off], E::mul(a, c)));
        d = E::mul(r, E::sub(D[off], E::mul(a, d)));
        c = E::mul(r, C[off]);
        Cs[off] = c;
        X[off] = d;
    }

    // Backward substitution: x_j = d'_j - c'_j x_{j+1}; x_{n-1} = d'_{n-1}.
    double x = d;
    bool finite = isfinite(x);
    j = n_row - 2;
    for (; j - THOMAS_UNR + 1 >= 0; j -= THOMAS_UNR) {
        double cs[THOMAS_UNR], ds[THOMAS_UNR];
#pragma unroll
        for (int u = 0; u < THOMAS_UNR; ++u) {
            size_t off = (size_t)(j - u) * ns + i;
            cs[u] = Cs[off];
            ds[u] = X[off];
        }
#pragma unroll
        for (int u = 0; u < THOMAS_UNR; ++u) {
            x = E::sub(ds[u], E::mul(cs[u], x));
            X[(size_t)(j - u) * ns + i] = x;
            finite &= isfinite(x);
        }
    }
    for (; j >= 0; --j) {
        size_t off = (size_t)j * ns + i;
        x = E::sub(X[off], E::mul(Cs[off], x));
        X[off] = x;
        finite &= isfinite(x);
    }
    if (!finite) raise_status(status, ST_NONFINITE);
}

// Periodic Thomas with the correction vector e (tdma_local.cpp:108-208).
// Needs n_row >= 3.  Cs holds c', Es holds e', X holds d' and then x.
__global__ void __launch_bounds__(THOMAS_BLOCK)
thomas_cyclic_f64_kernel(const double* __restrict__ A, const double* __restrict__ B,
                         const double* __restrict__ C, const double* D, double* X,
                         double* __restrict__ Cs, double* __restrict__ Es, int n_sys, int n_row,
                         unsigned* status) {
    using E = Exact64;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_sys) return;
    const size_t ns = (size_t)n_sys;
    const int nl = n_row - 1;

    // Row 1: e_1 = -A_1 scaled like d and c (row 0 is the periodic unknown).
    double inv_b = E::rcp(B[ns + i]);
    double d = E::mul(D[ns + i], inv_b);
    double e = E::mul(-A[ns + i], inv_b);
    double c = E::mul(C[ns + i], inv_b);
    Cs[ns + i] = c;
    Es[ns + i] = e;
    X[ns + i] = d;
    for (int j = 2; j <= nl; ++j) {
        size_t off = (size_t)j * ns + i;
        double a = A[off];
        double e0 = (j == nl) ? -C[off] : 0.0;  // e starts as -C_{n-1} at the last row
        double r = E::rcp(E::sub(B[off], E::mul(a, c)));
        d = E::mul(r, E::sub(D[off], E::mul(a, d)));
        e = E::mul(r, E::sub(e0, E::mul(a, e)));
        c = E::mul(r, C[off]);
        Cs[off] = c;
        Es[off] = e;
        X[off] = d;
    }
    const double d_last = d, e_last = e;
    for (int j = nl - 1; j >= 1; --j) {
        size_t off = (size_t)j * ns + i;
        double cj = Cs[off];
        d = E::sub(X[off], E::mul(cj, d));
        e = E::sub(Es[off], E::mul(cj, e));
        X[off] = d;
        Es[off] = e;
    }
    // d, e now hold row 1.
    const double a0 = A[i], c0 = C[i];
    const double x0 = E::div(E::sub(E::sub(D[i], E::mul(a0, d_last)), E::mul(c0, d)),
                             E::add(E::add(B[i], E::mul(a0, e_last)), E::mul(c0, e)));
    X[i] = x0;
    bool finite = isfinite(x0);
    for (int j = 1; j <= nl; ++j) {
        size_t off = (size_t)j * ns + i;
        double x = E::add(X[off], E::mul(x0, Es[off]));
        X[off] = x;
        finite &= isfinite(x);
    }
    if (!finite) raise_status(status, ST_NONFINITE);
}

}  // namespace btdma
