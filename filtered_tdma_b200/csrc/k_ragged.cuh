// Ragged batches: systems of different lengths stored back to back (CSR row
// offsets), each system contiguous.  Row j of system i is element off[i] + j of
// A, B, C, D and X.
//
// One group of P lanes (P a power of two <= 32) solves one system; a warp holds
// 32 / P groups.  The system is cut into P sub-segments (the reference's
// para_range split, libs/pascal_tdma/cpu/para_range.cpp:4-10), lane p owns
// sub-segment p and runs PaScaL's modified Thomas elimination on it
// (libs/pascal_tdma/cpu/pascal_tdma.cpp:131-170), reading its rows straight
// from global memory (consecutive rows of one lane share 32-byte sectors, which
// the L1 cache serves after the first miss) and keeping the per-row state in
// shared memory laid out [field][row][lane], so the 32 lanes of a warp touch 32
// consecutive doubles.  The reduced system of the P sub-segments is solved with
// warp shuffles (reduced_solve_shfl), then every lane back-substitutes its rows
// and stores x (FP64).
//
// The host sorts the systems into buckets of similar length (and separates
// periodic from non-periodic ones, so the shuffles of a warp are uniform); one
// launch per bucket, whose P and warps per CTA the autotuner picks.
#pragma once

#include "btdma_common.cuh"
#include "k_reduced.cuh"

namespace btdma {

struct RagArgs {
    const void* A;
    const void* B;
    const void* C;
    const void* D;
    double* X;
    const long long* off;  // [n_sys + 1] row offsets
    const int* list;       // systems of this bucket
    int count;             // entries of list
    int P;                 // lanes per system (power of two <= 32)
    int mcap;              // state slots per lane (>= longest sub-segment of the bucket)
    unsigned* status;
};

constexpr int RAG_LOOKAHEAD = 4;  // rows loaded ahead of the elimination

// Shared memory per warp: 3 fields x mcap rows x 32 lanes doubles.
__host__ __device__ __forceinline__ size_t rag_smem_bytes(int warps, int mcap) {
    return (size_t)warps * 3 * mcap * 32 * sizeof(double);
}

template <typename TIN, bool CYCLIC>
__global__ void __launch_bounds__(256) ragged_kernel(const RagArgs a) {
    extern __shared__ double rsm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int P = a.P;
    const int G = 32 / P;  // systems per warp
    const int g = lane / P;
    const int p = lane % P;
    const int mcap = a.mcap;
    double* st = rsm + (size_t)warp * 3 * mcap * 32 + lane;  // field f, row k: st[(f*mcap+k)*32]

    const int sidx = (blockIdx.x * (blockDim.x >> 5) + warp) * G + g;
    const bool have = sidx < a.count;
    int m = 0;
    long long row0 = 0;
    if (have) {
        const int sys = a.list[sidx];
        const long long o = a.off[sys];
        const int n = (int)(a.off[sys + 1] - o);
        const int base = n / P, rem = n % P;  // para_range: the first rem parts get one more row
        m = base + (p < rem ? 1 : 0);
        row0 = o + (long long)p * base + (p < rem ? p : rem);
    }
    const bool act = have && m >= 3;  // the host picks P <= n / 3
    const TIN* __restrict__ pA = static_cast<const TIN*>(a.A) + row0;
    const TIN* __restrict__ pB = static_cast<const TIN*>(a.B) + row0;
    const TIN* __restrict__ pC = static_cast<const TIN*>(a.C) + row0;
    const TIN* __restrict__ pD = static_cast<const TIN*>(a.D) + row0;

    // ------------------------------------------------------------ forward
    double ab0 = 0, cb0 = 0, db0 = 0;
    double alp = 0, gap = 0, dep = 0;  // row k-1
    double pi = 1.0, sa = 0.0, sd = 0.0, pi_last = 0.0;
    if (act) {
        for (int k0 = 0; k0 < m; k0 += RAG_LOOKAHEAD) {
            double ra[RAG_LOOKAHEAD], rb[RAG_LOOKAHEAD], rc[RAG_LOOKAHEAD], rd[RAG_LOOKAHEAD];
#pragma unroll
            for (int j = 0; j < RAG_LOOKAHEAD; ++j) {
                const int k = k0 + j < m ? k0 + j : m - 1;  // clamped (in bounds) tail loads
                ra[j] = (double)__ldg(pA + k);
                rb[j] = (double)__ldg(pB + k);
                rc[j] = (double)__ldg(pC + k);
                rd[j] = (double)__ldg(pD + k);
            }
#pragma unroll
            for (int j = 0; j < RAG_LOOKAHEAD; ++j) {
                const int k = k0 + j;
                if (k >= m) break;
                const double av = ra[j], bv = rb[j], cv = rc[j], dv = rd[j];
                double al, ga, de;
                if (k == 0) {
                    const double ib = rcp_nr(bv);
                    ab0 = av * ib;
                    cb0 = cv * ib;
                    db0 = dv * ib;
                    continue;
                } else if (k == 1) {
                    const double ib = rcp_nr(bv);
                    al = av * ib;
                    ga = cv * ib;
                    de = dv * ib;
                    sa = al;
                    sd = de;
                } else {
                    const double inv = rcp_nr(bv - av * gap);
                    ga = cv * inv;
                    de = (dv - av * dep) * inv;
                    al = -av * alp * inv;
                    if (k <= m - 2) {
                        pi = -gap * pi;
                        sa += pi * al;
                        sd += pi * de;
                    }
                }
                if (k == m - 1) pi_last = -gap * pi;
                st[(0 * mcap + k) * 32] = al;
                st[(1 * mcap + k) * 32] = ga;
                st[(2 * mcap + k) * 32] = de;
                alp = al;
                gap = ga;
                dep = de;
            }
        }
    }
    // reduced rows of this sub-segment (as in the tiled kernel)
    double l0 = 0, u0 = 0, r0 = 0, l1 = 0, u1 = 0, r1 = 0;
    if (act) {
        const double rr = rcp_nr(1.0 - cb0 * sa);
        l0 = rr * ab0;
        u0 = rr * cb0 * pi_last;
        r0 = rr * (db0 - cb0 * sd);
        l1 = alp;
        u1 = gap;
        r1 = dep;
    }
    double xf, xl;
    reduced_solve_shfl<CYCLIC>(l0, u0, r0, l1, u1, r1, p, P, P, act, xf, xl);

    // ------------------------------------------------ back substitution
    if (act) {
        double* xp = a.X + row0;
        double nonfinite = fma(xf, 0.0, fma(xl, 0.0, 0.0));
        xp[m - 1] = xl;
        double xn = xl;
        for (int k = m - 2; k >= 1; --k) {
            xn = st[(2 * mcap + k) * 32] - st[(0 * mcap + k) * 32] * xf -
                 st[(1 * mcap + k) * 32] * xn;
            nonfinite = fma(xn, 0.0, nonfinite);
            xp[k] = xn;
        }
        xp[0] = xf;
        if (nonfinite != 0.0) raise_status(a.status, ST_NONFINITE);  // NaN != 0
    }
}

}  // namespace btdma
