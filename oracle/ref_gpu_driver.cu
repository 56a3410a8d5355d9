// The reference's own GPU kernels on one GPU — TEST INFRASTRUCTURE ONLY.
//
// Built by `make -C oracle ref_gpu REF=<reference root>` into
// oracle/_ref/libref_gpu.so together with the reference's unmodified
// libs/pascal_tdma/gpu/tdma_local_cuda.cu; the Filtered kernels come from the
// reference's header libs/filtered_tdma/gpu/filtered_tdma_kernels.cuh, included
// unmodified.  Used by tests/test_reference_gpu.py (parity of these kernels
// with the oracle, so the emulation below is known to solve the same systems)
// and by bench.py's reference-GPU baseline leg (their time on the same B200 as
// the library's kernels).  The library never links or calls it.
//
// The reference splits a system's rows over P MPI ranks, one GPU each
// (PaScaLTDMACUDA::solve, libs/pascal_tdma/gpu/pascal_tdma_cuda.cu:266-287;
// FilteredTDMACUDA::solve_filtered_v2, libs/filtered_tdma/gpu/
// filtered_tdma_cuda.cu:158-196).  Here the P ranks' slabs are the P row blocks
// of one [n_row x n_sys] array on one GPU (rank q's slab starts at row r0_q,
// para_range split), every rank's kernels run in rank order on one stream, and
// the MPI transport is replaced by pointers:
//   PaScaL   — the ranks' reduced rows A_rd, B_rd, C_rd, D_rd are rows 2q and
//              2q+1 of one [2P x n_sys] array, which is then already the
//              reduced system the all-to-all would assemble; tdma_many_cuda
//              solves it, and each rank's update reads its two rows back.
//   Filtered — rank q's receive buffers are rank q-1's and q+1's send buffers.
// Arithmetic, launch shapes (block_x = 128, block_y = 1; FTDMA_BLOCK_SYS) and
// the order of kernels are the reference's.
#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "filtered_tdma_kernels.cuh"  // libs/filtered_tdma/gpu (static kernels)
#include "tdma_local_cuda.cuh"        // libs/pascal_tdma/gpu

namespace {

// para_range over [0, n): rank q owns rows [r0, r0 + m)
// (libs/pascal_tdma/cpu/para_range.cpp:4-10)
void split(int n, int P, int q, int* r0, int* m) {
    int base = n / P, rem = n % P;
    *r0 = q * base + (q < rem ? q : rem);
    *m = base + (q < rem ? 1 : 0);
}

struct Scratch {
    double* buf = nullptr;
    size_t cap = 0;
    int* J = nullptr;
    int Jcap = 0;
};
Scratch gp;  // PaScaL's reduced system
Scratch gf;  // Filtered rank state

int reserve(Scratch& g, size_t doubles, int nJ) {
    if (doubles > g.cap) {
        cudaFree(g.buf);
        g.buf = nullptr;
        g.cap = 0;
        if (cudaMalloc(&g.buf, doubles * sizeof(double)) != cudaSuccess) return -3;
        g.cap = doubles;
    }
    if (nJ > g.Jcap) {
        cudaFree(g.J);
        g.J = nullptr;
        g.Jcap = 0;
        if (cudaMalloc(&g.J, nJ * sizeof(int)) != cudaSuccess) return -3;
        g.Jcap = nJ;
    }
    return 0;
}

// Filtered rank state in the scratch buffer: per rank A_rho, C_rho [m + 1],
// then send_right, send_left [2 x n_sys] per rank; J per rank in g.J.
size_t filt_offsets(int n_sys, int n_row, int P, std::vector<size_t>& rho_off,
                           size_t* send_off) {
    size_t o = 0;
    rho_off.resize(P);
    for (int q = 0; q < P; ++q) {
        int r0, m;
        split(n_row, P, q, &r0, &m);
        rho_off[q] = o;
        o += 2 * (size_t)(m + 1);
    }
    *send_off = o;
    return o + (size_t)4 * P * n_sys;
}

}  // namespace

extern "C" {

// tdma_many_cuda (nprocs == 1: both libraries' solve): in place, D <- x.
int refgpu_tdma_many(double* A, double* B, double* C, double* D, int n_sys, int n_row,
                     cudaStream_t s) {
    tdma_many_cuda(A, B, C, D, n_sys, n_row, 128, 1, s);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// PaScaL with P ranks (every slab >= 3 rows): modified Thomas per rank, the
// reduced 2P-row system by tdma_many_cuda, the update per rank.  In place.
int refgpu_pascal(double* A, double* B, double* C, double* D, int n_sys, int n_row, int P,
                  cudaStream_t s) {
    const size_t nr = (size_t)2 * P * n_sys;
    if (reserve(gp, 4 * nr, 0)) return -3;
    double* Ard = gp.buf;
    double* Brd = Ard + nr;
    double* Crd = Brd + nr;
    double* Drd = Crd + nr;
    for (int q = 0; q < P; ++q) {
        int r0, m;
        split(n_row, P, q, &r0, &m);
        const size_t o = (size_t)r0 * n_sys, orow = (size_t)2 * q * n_sys;
        pascal_tdma_modified_thomas_cuda(A + o, B + o, C + o, D + o, Ard + orow, Brd + orow,
                                         Crd + orow, Drd + orow, n_sys, m, 128, 1, s);
    }
    tdma_many_cuda(Ard, Brd, Crd, Drd, n_sys, 2 * P, 128, 1, s);
    for (int q = 0; q < P; ++q) {
        int r0, m;
        split(n_row, P, q, &r0, &m);
        const size_t o = (size_t)r0 * n_sys, orow = (size_t)2 * q * n_sys;
        pascal_tdma_update_solution_cuda(A + o, C + o, D + o, Drd + orow, n_sys, m, 128, 1, s);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// k_set_rho on every rank's slab (FilteredTDMACUDA::set_rho_device, system 0's
// column); before the Filtered solves of a shape.
int refgpu_filtered_set_rho(const double* A, const double* B, const double* C, int n_sys,
                            int n_row, int P, cudaStream_t s) {
    std::vector<size_t> ro;
    size_t so;
    if (reserve(gf, filt_offsets(n_sys, n_row, P, ro, &so), P)) return -3;
    const Scratch& g = gf;
    for (int q = 0; q < P; ++q) {
        int r0, m;
        split(n_row, P, q, &r0, &m);
        const size_t o = (size_t)r0 * n_sys;
        double* Arho = g.buf + ro[q];
        double* Crho = Arho + (m + 1);
        k_set_rho<<<ftdma_grid1D(m + 1), FTDMA_BLOCK_SYS, 0, s>>>(Arho, Crho, A + o, B + o,
                                                                  C + o, n_sys, m);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

// solve_filtered_v2 on every rank (eps = eps_constant / (m P)^2, the
// constructor's rule with the rank's row count), the neighbour exchange by
// pointers.  In place; J of rank q into J_out[q] when J_out is non-null
// (blocking read).
int refgpu_filtered_v2(double* A, double* B, double* C, double* D, int n_sys, int n_row, int P,
                       double eps_constant, int* J_out, cudaStream_t s) {
    std::vector<size_t> ro;
    size_t so;
    const Scratch& g = gf;
    if (filt_offsets(n_sys, n_row, P, ro, &so) > g.cap || P > g.Jcap) return -1;
    const dim3 block(FTDMA_BLOCK_SYS);
    const dim3 grid = ftdma_grid1D(n_sys);
    auto send_right = [&](int q) { return g.buf + so + (size_t)(4 * q) * n_sys; };
    auto send_left = [&](int q) { return g.buf + so + (size_t)(4 * q + 2) * n_sys; };
    for (int q = 0; q < P; ++q) {
        int r0, m;
        split(n_row, P, q, &r0, &m);
        const size_t o = (size_t)r0 * n_sys;
        double* Arho = g.buf + ro[q];
        double* Crho = Arho + (m + 1);
        const double N = (double)m * P;
        const double eps = eps_constant / (N * N);
        double *a = A + o, *b = B + o, *c = C + o, *d = D + o;
        k_cal_J_rhs_bound<<<1, FTDMA_BLOCK_SYS, 0, s>>>(g.J + q, Arho, Crho, d,
                                                         d + (size_t)(m - 1) * n_sys, n_sys, m,
                                                         eps);
        k_fwd_pass_v2<<<grid, block, 0, s>>>(a, b, c, d, n_sys, m, g.J + q);
        k_bwd_pass_v2<<<grid, block, 0, s>>>(a, c, d, n_sys, m, g.J + q);
        k_pack_lastrow<<<grid, block, 0, s>>>(send_right(q), c, d, n_sys, m);
        k_pack_row0<<<grid, block, 0, s>>>(send_left(q), a, d, n_sys);
    }
    for (int q = 0; q < P; ++q) {
        int r0, m;
        split(n_row, P, q, &r0, &m);
        const size_t o = (size_t)r0 * n_sys;
        const double* rl = q > 0 ? send_right(q - 1) : send_right(q);
        const double* rr = q < P - 1 ? send_left(q + 1) : send_left(q);
        k_solve_both<<<grid, block, 0, s>>>(D + o, A + o, C + o, rl, rl + n_sys, rr,
                                            rr + n_sys, q > 0 ? 1 : 0, q < P - 1 ? 1 : 0,
                                            n_sys, m);
    }
    for (int q = 0; q < P; ++q) {
        int r0, m;
        split(n_row, P, q, &r0, &m);
        const size_t o = (size_t)r0 * n_sys;
        k_final_pass<<<grid, block, 0, s>>>(A + o, C + o, D + o, D + o,
                                            D + o + (size_t)(m - 1) * n_sys, n_sys, m,
                                            g.J + q);
    }
    if (cudaGetLastError() != cudaSuccess) return -3;
    if (J_out) {
        if (cudaMemcpyAsync(J_out, g.J, sizeof(int) * P, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return -3;
    }
    return 0;
}

// Kernel launches per solve, for the bench line.
int refgpu_launches(int method, int P) {
    if (method == 0) return 1;               // tdma_many
    if (method == 1) return 2 * P + 1;       // PaScaL
    return 7 * P;                            // Filtered v2
}

}  // extern "C"
