// HBM bandwidth of the row-interleaved access pattern as a function of the
// contiguous piece width.
//
// A system-batched array [n_row x n_sys] is contiguous only along systems, so
// a kernel that owns `w` consecutive systems reads every row as one piece of
// w * elem bytes, and consecutive pieces it reads are a whole row pitch apart.
// This probe streams A, B, C, D (elem = 4 or 8 bytes) and writes X (FP64) in
// pieces of 64..512 bytes with plain 16-byte vector loads and prints the
// achieved GB/s: the ceiling a solver with that piece width can reach, whatever
// its arithmetic.  Used by `python -m filtered_tdma_b200.width_probe`.
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

namespace {

template <int PW, typename T>
__global__ void __launch_bounds__(512) stream_pieces(const T* __restrict__ A, const T* __restrict__ B,
                                                     const T* __restrict__ C, const T* __restrict__ D,
                                                     double* __restrict__ X, int n_sys, int n_row) {
    constexpr int EPT = 16 / sizeof(T);  // elements per 16-byte vector
    constexpr int TPR = PW / 16;         // threads per row piece
    constexpr int RPI = 512 / TPR;       // rows per block iteration
    constexpr int SPB = PW / sizeof(T);  // systems per piece
    const int nblk = n_sys / SPB;
    for (int cb = blockIdx.x; cb < nblk; cb += gridDim.x) {
        const size_t col = (size_t)cb * SPB + (threadIdx.x % TPR) * EPT;
#pragma unroll 4
        for (int r = threadIdx.x / TPR; r < n_row; r += RPI) {
            const size_t o = (size_t)r * n_sys + col;
            const float4 a = *reinterpret_cast<const float4*>(A + o);
            const float4 b = *reinterpret_cast<const float4*>(B + o);
            const float4 c = *reinterpret_cast<const float4*>(C + o);
            const float4 d = *reinterpret_cast<const float4*>(D + o);
            if constexpr (sizeof(T) == 4) {
                double2* xp = reinterpret_cast<double2*>(X + o);
                xp[0] = make_double2((double)a.x + b.x + c.x + d.x, (double)a.y + b.y + c.y + d.y);
                xp[1] = make_double2((double)a.z + b.z + c.z + d.z, (double)a.w + b.w + c.w + d.w);
            } else {
                const double2 a2 = *reinterpret_cast<const double2*>(&a);
                const double2 b2 = *reinterpret_cast<const double2*>(&b);
                const double2 c2 = *reinterpret_cast<const double2*>(&c);
                const double2 d2 = *reinterpret_cast<const double2*>(&d);
                *reinterpret_cast<double2*>(X + o) =
                    make_double2(a2.x + b2.x + c2.x + d2.x, a2.y + b2.y + c2.y + d2.y);
            }
        }
    }
}

template <int PW, typename T>
int run(const void* buf[4], double* X, int n_sys, int n_row, int grid) {
    if (n_sys % (PW / (int)sizeof(T)) != 0) return 0;
    const T* A = static_cast<const T*>(buf[0]);
    const T* B = static_cast<const T*>(buf[1]);
    const T* C = static_cast<const T*>(buf[2]);
    const T* D = static_cast<const T*>(buf[3]);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 6; ++rep) {  // first launch is a warm-up
        cudaEventRecord(e0);
        stream_pieces<PW, T><<<grid, 512>>>(A, B, C, D, X, n_sys, n_row);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) return 1;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    const double bytes = (double)n_sys * n_row * (4 * sizeof(T) + 8);
    printf("{\"elem\": %d, \"piece_bytes\": %d, \"ms\": %.4f, \"gbs\": %.1f}\n", (int)sizeof(T), PW,
           best, bytes / best / 1e6);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    const int n_sys = argc > 1 ? atoi(argv[1]) : 262144;
    const int n_row = argc > 2 ? atoi(argv[2]) : 512;
    if (n_sys <= 0 || n_row <= 0 || n_sys % 128 != 0) {
        fprintf(stderr, "usage: width_probe [n_sys (multiple of 128)] [n_row]\n");
        return 2;
    }
    const size_t n = (size_t)n_sys * n_row;
    void* buf[5];
    for (auto& p : buf) {
        if (cudaMalloc(&p, n * 8) != cudaSuccess) {
            fprintf(stderr, "cudaMalloc failed\n");
            return 1;
        }
        cudaMemset(p, 0, n * 8);
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    const int grid = 4 * sms;
    const void* in[4] = {buf[0], buf[1], buf[2], buf[3]};
    double* X = static_cast<double*>(buf[4]);
    int rc = 0;
    rc |= run<64, float>(in, X, n_sys, n_row, grid);
    rc |= run<128, float>(in, X, n_sys, n_row, grid);
    rc |= run<256, float>(in, X, n_sys, n_row, grid);
    rc |= run<512, float>(in, X, n_sys, n_row, grid);
    rc |= run<64, double>(in, X, n_sys, n_row, grid);
    rc |= run<128, double>(in, X, n_sys, n_row, grid);
    rc |= run<256, double>(in, X, n_sys, n_row, grid);
    rc |= run<512, double>(in, X, n_sys, n_row, grid);
    const cudaError_t e = cudaDeviceSynchronize();
    if (rc || e != cudaSuccess) {
        fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e));
        return 1;
    }
    for (auto& p : buf) cudaFree(p);
    return 0;
}
