// Channel momentum ADI sweeps (apps/channel_gpu/MomentumSolverGPU.cu:135-220
// k_build_{x,y,z} + solve + k_scatter_{x,y,z}, called by adi_{z,y,x}_ at
// :261-313), with the coefficients generated inside the tiled solve (GEN = 3
// row tables) instead of stored: the build is a gather of the ghosted field
// into the sweep layout; the z and y sweeps store their solutions straight back
// into the field (the tiled solve's layout map), the x sweep through a
// transposing scatter.
//
// Field: q[i + (nx + 2) * (j + (ny + 2) * k)] (DeviceField.hpp df_idx), interior
// i = 1..nx, j = 1..ny, k = 1..nz.  Sweep layouts (system index fastest):
//   z: D[(k-1) * nx*ny + (j-1) * nx + (i-1)]     rows k, systems (j, i)
//   y: D[(j-1) * nx*nz + (k-1) * nx + (i-1)]     rows j, systems (k, i)
//   x: D[(i-1) * ny*nz + (k-1) * ny + (j-1)]     rows i, systems (k, j)
// (the reference orders the systems the other way round, s = (i-1) * ny +
// (j-1) etc.; a system's rows and coefficients are the same).
#pragma once

#include "btdma_common.cuh"

namespace btdma {

struct MomGeom {
    int nx, ny, nz;
};

__device__ __forceinline__ size_t mom_fld(const MomGeom& g, int i, int j, int k) {
    return (size_t)i + (size_t)(g.nx + 2) * ((size_t)j + (size_t)(g.ny + 2) * k);
}

// z and y sweeps: i fastest on both sides, no transpose.  pin: row k = 1 of
// the z sweep is the w wall (D = 0, k_build_z :150-152).  A block copies
// MOM_GR consecutive rows a (z: j, y: k) of one plane b, every load of a
// thread issued before its stores.  Grid (ceil(nx / 128), ceil(na / MOM_GR),
// nb), block 128.
constexpr int MOM_GR = 4;
template <int DIR>
__global__ void __launch_bounds__(128) mom_gather_kernel(const double* __restrict__ q,
                                                         double* __restrict__ D, const MomGeom g,
                                                         int pin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int a0 = blockIdx.y * MOM_GR + 1, b = blockIdx.z + 1;  // z: (j, k); y: (k, j)
    const int na = DIR == 2 ? g.ny : g.nz;
    if (i > g.nx) return;
    double v[MOM_GR];
#pragma unroll
    for (int r = 0; r < MOM_GR; ++r) {
        const int a = a0 + r;
        const int j = DIR == 2 ? a : b, k = DIR == 2 ? b : a;
        v[r] = a <= na ? q[mom_fld(g, i, j, k)] : 0.0;
    }
#pragma unroll
    for (int r = 0; r < MOM_GR; ++r) {
        const int a = a0 + r;
        if (a > na) break;
        const int j = DIR == 2 ? a : b, k = DIR == 2 ? b : a;
        const size_t o = DIR == 2 ? ((size_t)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1)
                                  : ((size_t)(j - 1) * g.nz + (k - 1)) * g.nx + (i - 1);
        D[o] = (DIR == 2 && pin && k == 1) ? 0.0 : v[r];
    }
}

// Inverse of mom_gather_kernel (z and y sweeps): the solution X in the sweep
// layout back into the field's interior.  Same grid and block.
template <int DIR>
__global__ void __launch_bounds__(128) mom_scatter_kernel(const double* __restrict__ X,
                                                          double* __restrict__ q,
                                                          const MomGeom g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int a0 = blockIdx.y * MOM_GR + 1, b = blockIdx.z + 1;  // z: (j, k); y: (k, j)
    const int na = DIR == 2 ? g.ny : g.nz;
    if (i > g.nx) return;
    double v[MOM_GR];
#pragma unroll
    for (int r = 0; r < MOM_GR; ++r) {
        const int a = a0 + r;
        const int j = DIR == 2 ? a : b, k = DIR == 2 ? b : a;
        const size_t o = DIR == 2 ? ((size_t)(k - 1) * g.ny + (j - 1)) * g.nx + (i - 1)
                                  : ((size_t)(j - 1) * g.nz + (k - 1)) * g.nx + (i - 1);
        v[r] = a <= na ? X[o] : 0.0;
    }
#pragma unroll
    for (int r = 0; r < MOM_GR; ++r) {
        const int a = a0 + r;
        if (a > na) break;
        const int j = DIR == 2 ? a : b, k = DIR == 2 ? b : a;
        q[mom_fld(g, i, j, k)] = v[r];
    }
}

// Explicit coefficients of one sweep for the array-based solvers (the
// Filtered backend), in the arithmetic and order of k_build_{x,y,z}
// (apps/channel_gpu/MomentumSolverGPU.cu:135-210): for row r with the axis
// factors ar, cr,  a = -c ar, cc = -c cr, b = 1 - a - cc; the z walls (one
// rank holds all of z): row 0 a = 0 and b += c ar, the last row cc = 0 and
// b += c cr (velocity components along the wall), or the w row 0 pinned to
// (0, 1, 0).  Every system of the sweep has the same rows.  Grid-stride over
// n_row x n_sys; round-to-nearest operations, no contraction.
__global__ void mom_coef_kernel(double* __restrict__ A, double* __restrict__ B,
                                double* __restrict__ C, const double* __restrict__ ar_,
                                const double* __restrict__ cr_, int n_row, int n_sys, double c,
                                int walls, int is_w) {
    const size_t n = (size_t)n_row * n_sys;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / (size_t)n_sys);
        const double ar = ar_[r], cr = cr_[r];
        double a = -__dmul_rn(c, ar), cc = -__dmul_rn(c, cr);
        double b = __dsub_rn(__dsub_rn(1.0, a), cc);
        if (walls && r == 0) {
            a = 0.0;
            if (!is_w) b = __dadd_rn(b, __dmul_rn(c, ar));
        }
        if (walls && r == n_row - 1) {
            cc = 0.0;
            if (!is_w) b = __dadd_rn(b, __dmul_rn(c, cr));
        }
        if (walls && is_w && r == 0) {
            a = 0.0;
            b = 1.0;
            cc = 0.0;
        }
        A[e] = a;
        B[e] = b;
        C[e] = cc;
    }
}

constexpr int MOM_TILE = 32;

// x sweep: (i, j) transposed through a shared 32 x 32 tile per k; block (32, 8).
__global__ void __launch_bounds__(256) mom_gather_x_kernel(const double* __restrict__ q,
                                                           double* __restrict__ D,
                                                           const MomGeom g) {
    __shared__ double tile[MOM_TILE][MOM_TILE + 1];
    const int i0 = blockIdx.x * MOM_TILE, j0 = blockIdx.y * MOM_TILE, k = blockIdx.z + 1;
#pragma unroll
    for (int u = 0; u < MOM_TILE / 8; ++u) {  // block (MOM_TILE, 8)
        const int r = threadIdx.y + 8 * u;
        const int i = i0 + threadIdx.x + 1, j = j0 + r + 1;
        if (i <= g.nx && j <= g.ny) tile[r][threadIdx.x] = q[mom_fld(g, i, j, k)];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < MOM_TILE / 8; ++u) {  // block (MOM_TILE, 8)
        const int r = threadIdx.y + 8 * u;
        const int j = j0 + threadIdx.x + 1, i = i0 + r + 1;
        if (i <= g.nx && j <= g.ny)
            D[((size_t)(i - 1) * g.nz + (k - 1)) * g.ny + (j - 1)] = tile[threadIdx.x][r];
    }
}

__global__ void __launch_bounds__(256) mom_scatter_x_kernel(const double* __restrict__ D,
                                                            double* __restrict__ q,
                                                            const MomGeom g) {
    __shared__ double tile[MOM_TILE][MOM_TILE + 1];
    const int j0 = blockIdx.x * MOM_TILE, i0 = blockIdx.y * MOM_TILE, k = blockIdx.z + 1;
#pragma unroll
    for (int u = 0; u < MOM_TILE / 8; ++u) {  // block (MOM_TILE, 8)
        const int r = threadIdx.y + 8 * u;
        const int j = j0 + threadIdx.x + 1, i = i0 + r + 1;
        if (i <= g.nx && j <= g.ny)
            tile[r][threadIdx.x] = D[((size_t)(i - 1) * g.nz + (k - 1)) * g.ny + (j - 1)];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < MOM_TILE / 8; ++u) {  // block (MOM_TILE, 8)
        const int r = threadIdx.y + 8 * u;
        const int i = i0 + threadIdx.x + 1, j = j0 + r + 1;
        if (i <= g.nx && j <= g.ny) q[mom_fld(g, i, j, k)] = tile[threadIdx.x][r];
    }
}

}  // namespace btdma
