// Driver for the reference's channel-flow coefficient-build kernels —
// TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile (`make ref_channel REF=<reference root>`) compiles the
// reference's apps/channel_gpu/MomentumSolverGPU.cu and PressureSolverGPU.cu
// unmodified (the reference's NVCCFLAGS, sm_100a, the MPI stand-in of
// mpi_shim/) and links them with this file into _ref/libref_channel.so.  Only
// the kernels declared below are launched: the solver classes around them
// (MPI transposes, cuFFT plans, the TDMA objects) are never constructed, and
// their unresolved symbols stay unbound (the library is loaded with
// RTLD_LAZY).  The declarations repeat the kernels' signatures so that these
// launches bind to the reference's own kernel stubs:
//   MomentumSolverGPU.cu:135-220 (k_build_{z,y,x}, k_scatter_{z,y,x})
//   PressureSolverGPU.cu:183-234 (k_build_poisson_tdma, k_zero_mode,
//                                 k_write_poisson_solution)
// The library is used by tests/ to pin oracle/momentum_oracle.py and
// oracle/poisson_oracle.py; nothing in the product links it.

#include <cuComplex.h>
#include <cuda_runtime.h>

typedef cuDoubleComplex cufftDoubleComplex;

namespace channel {
namespace gpu_kernels {
__global__ void k_build_z(int comp, const double* q, double* A, double* B, double* C, double* D,
                          const double* dz, const double* dmz, int nx, int ny, int nz, double c,
                          int low, int high);
__global__ void k_scatter_z(const double* D, double* q, int nx, int ny, int nz);
__global__ void k_build_y(int comp, const double* q, double* A, double* B, double* C, double* D,
                          const double* dy, const double* dmy, int nx, int ny, int nz, double c);
__global__ void k_scatter_y(const double* D, double* q, int nx, int ny, int nz);
__global__ void k_build_x(int comp, const double* q, double* A, double* B, double* C, double* D,
                          const double* dx, const double* dmx, int nx, int ny, int nz, double c);
__global__ void k_scatter_x(const double* D, double* out, int nx, int ny, int nz);
__global__ void k_build_poisson_tdma(const cufftDoubleComplex* hat_Y, double* Am, double* Ac,
                                     double* Ap, double* Am2, double* Ac2, double* Ap2,
                                     double* Br, double* Bi, const double* dzg,
                                     const double* dmzg, const double* kx2, const double* ky2,
                                     int n3I, int nsys, int hme, int n2m, int ix0, int rank_xz,
                                     int size_xz);
__global__ void k_zero_mode(double* Am, double* Ac, double* Ap, double* Am2, double* Ac2,
                            double* Ap2, double* Br, double* Bi);
__global__ void k_write_poisson_solution(cufftDoubleComplex* hat_Y, const double* Br,
                                         const double* Bi, int n3I, int nsys, int hme, int n2m);
}  // namespace gpu_kernels
}  // namespace channel

using namespace channel::gpu_kernels;

namespace {
constexpr int kBlock = 256;  // the reference's launch block (MomentumSolverGPU.cu:261-313)
int grid_for(long n) { return (int)((n + kBlock - 1) / kBlock); }
int finish() {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}
}  // namespace

extern "C" {

// One momentum sweep's build (direction 0 = x, 1 = y, 2 = z) as
// MomentumSolverGPU::adi_{x,y,z}_ launches it; device pointers.  The z build
// takes the wall flags (low, high) of the one-rank case.
int refch_build(int dir, int comp, const double* q, double* A, double* B, double* C, double* D,
                const double* d, const double* dm, int nx, int ny, int nz, double c, int low,
                int high) {
    const long n = (long)nx * ny * nz;
    if (dir == 2)
        k_build_z<<<grid_for(n), kBlock>>>(comp, q, A, B, C, D, d, dm, nx, ny, nz, c, low, high);
    else if (dir == 1)
        k_build_y<<<grid_for(n), kBlock>>>(comp, q, A, B, C, D, d, dm, nx, ny, nz, c);
    else
        k_build_x<<<grid_for(n), kBlock>>>(comp, q, A, B, C, D, d, dm, nx, ny, nz, c);
    return finish();
}

int refch_scatter(int dir, const double* D, double* q, int nx, int ny, int nz) {
    const long n = (long)nx * ny * nz;
    if (dir == 2)
        k_scatter_z<<<grid_for(n), kBlock>>>(D, q, nx, ny, nz);
    else if (dir == 1)
        k_scatter_y<<<grid_for(n), kBlock>>>(D, q, nx, ny, nz);
    else
        k_scatter_x<<<grid_for(n), kBlock>>>(D, q, nx, ny, nz);
    return finish();
}

// PressureSolverGPU::solve_tdma_z_'s build and mode-(0,0) pin on one rank
// (rank_xz = 0, size_xz = 1, ix0 = 0, hme = the x modes held, n2m = ny).
int refch_poisson_build(const void* hat_Y, double* Am, double* Ac, double* Ap, double* Am2,
                        double* Ac2, double* Ap2, double* Br, double* Bi, const double* dzg,
                        const double* dmzg, const double* kx2, const double* ky2, int n3, int nsys,
                        int hme, int n2m, int pin) {
    const long n = (long)n3 * nsys;
    k_build_poisson_tdma<<<grid_for(n), kBlock>>>(
        static_cast<const cufftDoubleComplex*>(hat_Y), Am, Ac, Ap, Am2, Ac2, Ap2, Br, Bi, dzg,
        dmzg, kx2, ky2, n3, nsys, hme, n2m, 0, 0, 1);
    if (pin) k_zero_mode<<<1, 1>>>(Am, Ac, Ap, Am2, Ac2, Ap2, Br, Bi);
    return finish();
}

int refch_poisson_write(void* hat_Y, const double* Br, const double* Bi, int n3, int nsys, int hme,
                        int n2m) {
    const long n = (long)n3 * nsys;
    k_write_poisson_solution<<<grid_for(n), kBlock>>>(static_cast<cufftDoubleComplex*>(hat_Y), Br,
                                                      Bi, n3, nsys, hme, n2m);
    return finish();
}

}  // extern "C"
