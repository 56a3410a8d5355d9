// One theta-scheme ADI step of the reference's 3-D heat application
// (apps/heat_gpu/solve_theta.cu:121-351 and its step loop at :499-600), fused
// around the constant-coefficient tiled solve.
//
// Grid: ix x iy x iz interior cells on [-1, 1]^3 with one ghost layer; theta is
// the full grid, theta[(k * ny + j) * nx + i], nx = ix + 2 (i = ii + 1 for
// interior index ii).  Stencil per direction (stencil_coeffs.hpp:10-13):
// base = dt / (2 dd^2), a = c = base, b = -2 base.  Dirichlet walls use the
// reflection ghost u_ghost = 2 u_BC - u_adjacent (mpi_subdomain.cpp boundary()),
// folded fully implicitly: the wall row of each sweep gets base more on the
// diagonal and base * (ghost + adjacent) on the right-hand side
// (solve_theta.cu:185-201).
//
// Differences from the reference's kernel sequence, none of which changes the
// arithmetic of a cell:
//   * ghosts are not stored: a stencil neighbour outside the interior is
//     computed as 2 u_BC - theta(cell), exactly the value the reference's ghost
//     kernels write there;
//   * A, B, C are never materialised (the solve generates them);
//   * the right-hand side of the step (all directions' explicit half and the
//     Z wall folds) is computed inside the Z sweep from theta (the tiled
//     solve's GEN 4 mode, k_tile.cuh), so it is never stored; heat_rhs_z_kernel
//     below remains for Z sweeps that mode does not take (fewer than 2 or
//     more than 32 sub-segments);
//   * the Z sweep stores its solution straight into the Y sweep's layout
//     ([kk][jj][ii] -> [jj][kk][ii], the tiled solve's mapped store; the Y wall
//     folds then touch the two wall planes only), and the X sweep straight
//     into theta (its rows are contiguous there: the tiled solve stages each
//     group's solution in shared memory and stores it coalesced; storing it
//     row by row from the lanes, rows 2 KB apart, was slower than a separate
//     transpose); the Y sweep stores into the X sweep's layout the same way,
//     and the X wall folds touch the two wall planes.  heat_y_to_x_kernel
//     (a transpose through shared-memory tiles) remains for Y sweeps whose
//     staged store does not fit.
#pragma once

#include "btdma_common.cuh"

namespace btdma {

struct HeatGeom {
    int ix, iy, iz;        // interior cells
    double dt;
    double bx, by, bz;     // stencil base per direction: dt / (2 dd^2)
    const double* xc;      // cell centres incl. ghosts [ix + 2]
    const double* yc;      // [iy + 2]
    const double* zc;      // [iz + 2]
    const double* cx;      // cos(pi xc) [ix + 2] (host-computed once)
    const double* cy;      // cos(pi yc) [iy + 2]
    const double* cz;      // cos(pi zc) [iz + 2]
};

__device__ __forceinline__ size_t heat_full(const HeatGeom& g, int i, int j, int k) {
    return ((size_t)k * (g.iy + 2) + j) * (g.ix + 2) + i;
}

constexpr double HEAT_PI = 3.14159265358979323846;

// Right-hand side of the step (all directions' explicit half) plus the Z wall
// folds, written in the Z-sweep layout D[(kk * iy + jj) * ix + ii]
// (solve_theta.cu:121-160 and build_lhs_z_kernel :168-202).
// 2.5-D: a thread owns column (ii, jj) and walks HEAT_KCH planes, keeping
// theta at k - 1, k, k + 1 in registers; the x neighbours come from the
// adjacent lanes (warp shuffles; the warp's edge lanes load theirs), the y
// neighbours from the adjacent rows.  Block (128), grid (ix / 128, iy,
// iz / HEAT_KCH).  Lanes past the row (ix % 32 == 16) take part in the
// shuffles on the last column's values and store nothing; a live lane never
// uses a dead neighbour (its x neighbour past the row is the wall ghost).
constexpr int HEAT_KCH = 16;
__global__ void __launch_bounds__(128) heat_rhs_z_kernel(const double* __restrict__ theta,
                                                         double* __restrict__ D,
                                                         const HeatGeom g) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int jj = blockIdx.y;
    const int k0 = blockIdx.z * HEAT_KCH;  // first interior plane kk of this block
    const int lane = threadIdx.x & 31;
    if (ii - lane >= g.ix) return;         // the whole warp is past the row
    const bool live = ii < g.ix;
    const int i = (live ? ii : g.ix - 1) + 1, j = jj + 1;
    const int sy = g.ix + 2;                 // j stride of the full grid
    const int sz = (g.iy + 2) * (g.ix + 2);  // k stride (< 2^31 for grids this library takes)
    const double cxi = g.cx[i], cyj = g.cy[j];
    const double* col = theta + heat_full(g, i, j, 0);  // this column at k = 0
    // theta at k - 1 and k for the first plane (k = k0 + 1)
    double tm = col[(size_t)k0 * sz], t = col[(size_t)(k0 + 1) * sz];
    for (int kk = k0; kk < k0 + HEAT_KCH; ++kk) {  // iz % HEAT_KCH == 0 (btdma_heat_create)
        const int k = kk + 1;
        const double* c0 = col + (size_t)k * sz;
        const double tn = c0[sz];  // theta(k + 1): a ghost plane at the top wall, not read
        const double czk = g.cz[k];
        double tip, tim, tjp, tjm, tkp, tkm;
        {
            const double ubc = -cyj * czk;  // x walls
            double right = __shfl_down_sync(0xffffffffu, t, 1);
            double left = __shfl_up_sync(0xffffffffu, t, 1);
            if (lane == 31) right = live && ii + 1 < g.ix ? c0[1] : 0.0;
            if (lane == 0) left = ii > 0 ? c0[-1] : 0.0;
            tip = ii + 1 < g.ix ? right : 2.0 * ubc - t;
            tim = ii > 0 ? left : 2.0 * ubc - t;
        }
        {
            const double ubc = -cxi * czk;  // y walls
            tjp = jj + 1 < g.iy ? c0[sy] : 2.0 * ubc - t;
            tjm = jj > 0 ? c0[-sy] : 2.0 * ubc - t;
        }
        const double ubz = -cxi * cyj;  // z walls
        tkp = kk + 1 < g.iz ? tn : 2.0 * ubz - t;
        tkm = kk > 0 ? tm : 2.0 * ubz - t;
        const double src = g.dt * 3.0 * HEAT_PI * HEAT_PI * cxi * cyj * czk;
        double rhs = (g.bx * tip + g.bx * tim) + (g.by * tjp + g.by * tjm) +
                     (g.bz * tkp + g.bz * tkm) +
                     (1.0 + (-2.0 * g.bx) + (-2.0 * g.by) + (-2.0 * g.bz)) * t + src;
        // fully implicit Z walls: base * (ghost + boundary cell) to the right-hand side
        if (kk == 0) rhs += g.bz * ((2.0 * ubz - t) + t);
        if (kk == g.iz - 1) rhs += g.bz * ((2.0 * ubz - t) + t);
        if (live) D[((size_t)kk * g.iy + jj) * g.ix + ii] = rhs;
        tm = t;
        t = tn;
    }
}

// Y wall folds on the Z solution, already in the Y-sweep layout [jj][kk][ii]
// (build_lhs_y_kernel's right-hand-side terms, solve_theta.cu:205-253): planes
// jj = 0 and jj = iy - 1 get base * (ghost + boundary cell).  Grid (ix / 128,
// 2, iz).
__global__ void __launch_bounds__(128) heat_y_fold_kernel(const double* __restrict__ theta,
                                                          double* __restrict__ Dy,
                                                          const HeatGeom g) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int jj = blockIdx.y == 0 ? 0 : g.iy - 1;
    const int kk = blockIdx.z;
    if (ii >= g.ix) return;
    const int i = ii + 1, k = kk + 1, j = jj + 1;
    const double t = theta[heat_full(g, i, j, k)];
    const double ubc = -g.cx[i] * g.cz[k];
    Dy[((size_t)jj * g.iz + kk) * g.ix + ii] += g.by * ((2.0 * ubc - t) + t);
}

// X wall folds on the Y solution, already in the X-sweep layout [ii][kk][jj]
// (build_lhs_x_kernel's right-hand-side terms, solve_theta.cu:256-332): planes
// ii = 0 and ii = ix - 1 get base * (ghost + boundary cell), added to the
// value as heat_y_to_x_kernel adds it.  Grid (iy / 128, 2, iz).
__global__ void __launch_bounds__(128) heat_x_fold_kernel(const double* __restrict__ theta,
                                                          double* __restrict__ Dx,
                                                          const HeatGeom g) {
    const int jj = blockIdx.x * blockDim.x + threadIdx.x;
    const int ii = blockIdx.y == 0 ? 0 : g.ix - 1;
    const int kk = blockIdx.z;
    if (jj >= g.iy) return;
    const int i = ii + 1, j = jj + 1, k = kk + 1;
    const double t = theta[heat_full(g, i, j, k)];
    const double ubc = -g.cy[j] * g.cz[k];
    Dx[((size_t)ii * g.iz + kk) * g.iy + jj] += g.bx * ((2.0 * ubc - t) + t);
}

constexpr int HEAT_TILE = 32;

// Y solution [jj][kk][ii] -> X-sweep layout [ii][kk][jj] plus the X wall folds
// (copy_y_to_rhs + build_lhs_x_kernel, solve_theta.cu:256-332), through a
// shared 32 x 32 tile so both sides are coalesced.  Block (32, 8).
__global__ void __launch_bounds__(256) heat_y_to_x_kernel(const double* __restrict__ theta,
                                                          const double* __restrict__ Dy,
                                                          double* __restrict__ Dx,
                                                          const HeatGeom g) {
    __shared__ double tile[HEAT_TILE][HEAT_TILE + 1];
    const int ii0 = blockIdx.x * HEAT_TILE, jj0 = blockIdx.y * HEAT_TILE, kk = blockIdx.z;
#pragma unroll
    for (int u = 0; u < HEAT_TILE / 8; ++u) {  // block (HEAT_TILE, 8)
        const int r = threadIdx.y + 8 * u;
        const int ii = ii0 + threadIdx.x, jj = jj0 + r;
        if (ii < g.ix && jj < g.iy) tile[r][threadIdx.x] = Dy[((size_t)jj * g.iz + kk) * g.ix + ii];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < HEAT_TILE / 8; ++u) {  // block (HEAT_TILE, 8)
        const int r = threadIdx.y + 8 * u;
        const int jj = jj0 + threadIdx.x, ii = ii0 + r;
        if (ii < g.ix && jj < g.iy) {
            double v = tile[threadIdx.x][r];
            if (ii == 0 || ii == g.ix - 1) {
                const int j = jj + 1, k = kk + 1, i = ii == 0 ? 1 : g.ix;
                const double t = theta[heat_full(g, i, j, k)];
                const double ubc = -g.cy[j] * g.cz[k];
                if (ii == 0) v += g.bx * ((2.0 * ubc - t) + t);
                if (ii == g.ix - 1) v += g.bx * ((2.0 * ubc - t) + t);
            }
            Dx[((size_t)ii * g.iz + kk) * g.iy + jj] = v;
        }
    }
}

// Initial field on the full grid, ghosts included (mpi_subdomain.cpp
// initialization): sin(pi x) sin(pi y) sin(pi z) + cos(pi x) cos(pi y) cos(pi z).
__global__ void heat_init_kernel(double* __restrict__ theta, const HeatGeom g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= g.ix + 2) return;
    const double x = g.xc[i], y = g.yc[j], z = g.zc[k];
    theta[heat_full(g, i, j, k)] = sin(HEAT_PI * x) * sin(HEAT_PI * y) * sin(HEAT_PI * z) +
                                   cos(HEAT_PI * x) * cos(HEAT_PI * y) * cos(HEAT_PI * z);
}

// Sum over interior cells of (theta - exact)^2 with the manufactured solution
// exact = sin sin sin * exp(-3 pi^2 t) + cos cos cos (heat_cpu/main.cpp:59-79).
__global__ void heat_err_kernel(const double* __restrict__ theta, const HeatGeom g, double decay,
                                double* __restrict__ sum) {
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    const int jj = blockIdx.y, kk = blockIdx.z;
    double e = 0.0;
    if (ii < g.ix) {
        const int i = ii + 1, j = jj + 1, k = kk + 1;
        const double x = g.xc[i], y = g.yc[j], z = g.zc[k];
        const double ex = sin(HEAT_PI * x) * sin(HEAT_PI * y) * sin(HEAT_PI * z) * decay +
                          cos(HEAT_PI * x) * cos(HEAT_PI * y) * cos(HEAT_PI * z);
        const double d = theta[heat_full(g, i, j, k)] - ex;
        e = d * d;
    }
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, e);
}

}  // namespace btdma
