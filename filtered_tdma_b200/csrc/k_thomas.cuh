// Serial Thomas kernels (P = 1): one thread per system, row-interleaved layout.
//
// Bit-identical to the reference's CPU tdma_many / tdma_cyclic_many
// (libs/pascal_tdma/cpu/tdma_local.cpp:6-52, 108-208): the same operation order,
// IEEE round-to-nearest for every operation, no fused multiply-add (the
// reference's CPU build does not contract).  The reference's own GPU kernel
// divides row 0 by B instead of multiplying by 1/B
// (libs/pascal_tdma/gpu/tdma_local_cuda.cu:43-44), so it is not the bit oracle.
//
// thomas_f64_kernel: the forward sweep keeps the running (c', d') in registers
// and spills c' to the handle's scratch and d' to X; the backward sweep reads
// them back.  thomas_staged_kernel (short systems) keeps both on chip.  Loads are
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

// Staged serial Thomas for short systems (n_row <= THOMAS_STAGED_MAX_ROWS),
// bit-identical to thomas_f64_kernel and to tdma_many, at the algorithmic
// 40 B/row: one warp per CTA owns 32 consecutive systems; their C and D rows
// come into shared memory by TMA in chunks of 16 rows (one mbarrier per chunk,
// so the sweep starts on the first chunk), and the sweep overwrites them with
// c' and d' and then x in place — the scratch never leaves the chip
// (thomas_f64_kernel writes c' and d' to HBM and reads them back: 72 B/row).
// A and B go straight from HBM into registers, a chunk ahead of the sweep.
// x leaves by TMA stores of the D tile.  Rows past n_row and systems past
// n_sys in the last chunk / CTA are zero-filled by the loads and clipped by
// the stores.  Needs 16-byte aligned C, D, X and an even n_sys (TMA).
constexpr int THOMAS_STAGED_MAX_ROWS = 128;
constexpr int THOMAS_STAGED_SYS = 32;
constexpr int THOMAS_STAGED_CHUNK = 16;

__host__ __device__ __forceinline__ size_t thomas_staged_smem_bytes(int n_row) {
    const int nch = (n_row + THOMAS_STAGED_CHUNK - 1) / THOMAS_STAGED_CHUNK;
    return 2ull * nch * THOMAS_STAGED_CHUNK * THOMAS_STAGED_SYS * sizeof(double) +
           (size_t)nch * sizeof(uint64_t) + 128;
}

__global__ void __launch_bounds__(THOMAS_STAGED_SYS)
thomas_staged_kernel(const __grid_constant__ CUtensorMap tmC,
                     const __grid_constant__ CUtensorMap tmD,
                     const __grid_constant__ CUtensorMap tmX, const double* __restrict__ A,
                     const double* __restrict__ B, int n_sys, int n_row, unsigned* status) {
    using E = Exact64;
    constexpr int S = THOMAS_STAGED_SYS, CH = THOMAS_STAGED_CHUNK;
    extern __shared__ unsigned char smem_raw[];
    double* TC = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const int nch = (n_row + CH - 1) / CH;
    double* TD = TC + (size_t)nch * CH * S;
    uint64_t* bars = reinterpret_cast<uint64_t*>(TD + (size_t)nch * CH * S);
    const int s = threadIdx.x;
    const int g = blockIdx.x;
    const int sys = g * S + s;
    const bool valid = sys < n_sys;
    const size_t ns = (size_t)n_sys;

    if (s == 0) {
        for (int c = 0; c < nch; ++c) mbar_init(&bars[c], 1);
        fence_mbar_init();
    }
    __syncwarp();
    if (s == 0) {
        for (int c = 0; c < nch; ++c) {
            mbar_expect_tx(&bars[c], 2u * CH * S * sizeof(double));
            tma_load_2d(TC + (size_t)c * CH * S, &tmC, g * S, c * CH, &bars[c]);
            tma_load_2d(TD + (size_t)c * CH * S, &tmD, g * S, c * CH, &bars[c]);
        }
    }
    // A and B of chunk c into registers (0 and 1 outside the batch)
    auto load_ab = [&](int c, double (&a)[CH], double (&b)[CH]) {
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int j = c * CH + u;
            const bool in = valid && j < n_row;
            a[u] = in ? __ldg(A + (size_t)j * ns + sys) : 0.0;
            b[u] = in ? __ldg(B + (size_t)j * ns + sys) : 1.0;
        }
    };
    double ac[CH], bc[CH], an[CH], bn[CH];
    load_ab(0, ac, bc);
    if (nch > 1) load_ab(1, an, bn);
    bool ok = mbar_wait_bounded(&bars[0], 0, status);
#define TS(Z, j) Z[(size_t)(j) * S + s]
    // row 0: inv = 1/B, d = D inv, c = C inv (tdma_local.cpp:17-22)
    double c, d;
    {
        const double inv_b = E::rcp(bc[0]);
        d = E::mul(TS(TD, 0), inv_b);
        c = E::mul(TS(TC, 0), inv_b);
        TS(TD, 0) = d;
        TS(TC, 0) = c;
    }
    for (int ch = 0; ch < nch; ++ch) {
        if (ch > 0) {
#pragma unroll
            for (int u = 0; u < CH; ++u) {
                ac[u] = an[u];
                bc[u] = bn[u];
            }
            if (ch + 1 < nch) load_ab(ch + 1, an, bn);
            if (ok) ok = mbar_wait_bounded(&bars[ch], 0, status);
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int j = ch * CH + u;
            if (j == 0 || j >= n_row) continue;
            const double a = ac[u];
            const double r = E::rcp(E::sub(bc[u], E::mul(a, c)));
            d = E::mul(r, E::sub(TS(TD, j), E::mul(a, d)));
            c = E::mul(r, TS(TC, j));
            TS(TD, j) = d;
            TS(TC, j) = c;
        }
    }
    // backward substitution: x_j = d'_j - c'_j x_{j+1}; x_{n-1} = d'_{n-1}
    double x = d;
    bool finite = isfinite(x);
#pragma unroll 8
    for (int j = n_row - 2; j >= 0; --j) {
        x = E::sub(TS(TD, j), E::mul(TS(TC, j), x));
        TS(TD, j) = x;
        finite &= isfinite(x);
    }
#undef TS
    if (valid && !finite) raise_status(status, ST_NONFINITE);
    fence_async_shared();
    __syncwarp();
    if (s == 0) {
        for (int c2 = 0; c2 < nch; ++c2)
            tma_store_2d(&tmX, g * S, c2 * CH, TD + (size_t)c2 * CH * S);
        tma_store_commit();
        tma_store_wait_read();
    }
    if (!ok) {
        // a chunk wait gave up: one more bounded chance for the copies to land
        // before this CTA's shared memory is released
        if (s == 0)
            for (int c2 = 0; c2 < nch; ++c2) mbar_wait_bounded(&bars[c2], 0, nullptr, 1u << 16);
    }
    __syncwarp();
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
