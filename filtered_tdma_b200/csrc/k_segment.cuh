// Segmented solves (P >= 2): PaScaL and Filtered v1/v2 inside one GPU.
//
// The reference splits each system's rows over P MPI ranks
// (libs/pascal_tdma/cpu/pascal_tdma.cpp, libs/filtered_tdma/cpu/filtered_tdma.cpp).
// Here the P segments of a group of SEG_S systems are the P CTAs of one
// thread-block cluster:
//
//   * CTA k of the cluster owns rows [r0_k, r0_k + m_k) (para_range split) of
//     systems [g*SEG_S, (g+1)*SEG_S); one thread per system.
//   * The segment tile (A, B, C, D: 4 * m * SEG_S doubles) is staged once into
//     shared memory by TMA in chunks of SEG_BOXR rows, each chunk completing on
//     its own mbarrier, so the forward sweep starts on the first chunk while the
//     others are still in flight.  Filtered streams B instead (only the forward
//     sweep reads it): straight from HBM, a chunk ahead into registers, and
//     holds the first SEG_REG rows of each segment (inputs, then state) in
//     registers when every segment has SEG_REG + 2 rows or more, so its tile
//     has three arrays of m - SEG_REG rows (5 CTAs per SM at 64 rows instead of
//     3).  PaScaL keeps B staged (the tile's B part holds its reduced-system
//     scratch afterwards) and the first SEG_REG rows in registers on the same
//     condition (4 CTAs per SM).  A, B, C, D are read from HBM exactly once.
//   * The modified Thomas sweeps run in place on the tile (the reference's
//     per-rank steps, pascal_tdma.cpp:131-183 / filtered_tdma_kernels.hpp:35-189,
//     with the same operation order, IEEE round-to-nearest, no FMA).
//   * Each CTA publishes its two reduced rows in shared memory; the cluster
//     barrier replaces the reference's MPI exchange, and the neighbours' rows are
//     read directly through distributed shared memory:
//       PaScaL   — every CTA solves the whole 2P-row reduced system for its
//                  systems (the reference's all-to-all + tdma_many on the
//                  transposed reduced system, pascal_tdma.cpp:185-210);
//       Filtered — each CTA solves its two adjacent 2x2 interface systems
//                  (filtered_tdma_kernels.hpp:197-218).
//   * The final update (full for PaScaL, J-truncated for Filtered) runs on the
//     tile and x is written back with TMA stores: the only HBM write.
//
// HBM traffic: 32 B read + 8 B written per row, plus boxes rounded up to whole
// chunks at segment ends.  Without TMA (odd n_sys or unaligned pointers) the tile
// is filled and drained with coalesced per-thread loads and stores instead.
#pragma once

#include <cooperative_groups.h>

#include "btdma_common.cuh"

namespace btdma {

namespace cg = cooperative_groups;

constexpr int SEG_S = 32;     // systems per CTA (one warp; a 256-byte TMA box row)
constexpr int SEG_BOXR = 16;  // rows per TMA chunk
constexpr int SEG_MAX_P = 16; // cluster size limit (non-portable above 8)
constexpr int SEG_REG = 16;   // leading rows of a segment held in registers
static_assert(SEG_REG % SEG_BOXR == 0, "tile chunks start on a chunk boundary of the segment");

enum SegMethod { SEG_PASCAL = 0, SEG_FILT_V1 = 1, SEG_FILT_V2 = 2 };

// v1 runs the kernel twice: once to obtain the post-interface boundary values
// from which J is estimated, once to apply the correction with that J.
enum SegMode { SEG_MODE_SOLVE = 0, SEG_MODE_INTERFACE = 1 };

struct SegArgs {
    const double* A;
    const double* B;
    const double* C;
    const double* D;
    double* X;
    int n_sys, n_row, P;
    int mcap;      // tile rows per array (multiple of SEG_BOXR)
    int use_tma;   // tensor maps valid
    int mode;      // SegMode
    const int* J;  // Filtered: J per segment (device)
    unsigned long long* bnd;  // v1 interface pass: per segment max |x0|, max |xN| (bits)
    unsigned* status;
    // gate (optional): the launch runs only when (*gate != 0) == gate_run; a
    // Filtered solve and its exact fallback are launched back to back and one
    // of them does nothing (the device decides, no host round trip)
    const unsigned* gate;
    int gate_run;
};

// Dynamic shared memory layout of one CTA: the tiles (A, B, C, D for PaScaL;
// A, C, D for Filtered), the published reduced rows, PaScaL's reduced-solve
// scratch (in the B tile, dead after the forward sweep, whenever it fits there)
// and the chunk barriers.
__host__ __device__ __forceinline__ size_t seg_rsc_bytes(int P, bool cyclic) {
    return (cyclic ? 4ull : 3ull) * 2 * P * SEG_S * sizeof(double);
}
// mt: tile rows (the B tile's capacity)
__host__ __device__ __forceinline__ bool seg_rsc_in_b(int mt, int P, bool cyclic) {
    return seg_rsc_bytes(P, cyclic) <= (size_t)mt * SEG_S * sizeof(double);
}
// Tile rows of a segment of mcap rows, rr of them held in registers: rounded up
// to whole TMA chunks (every chunk lands as SEG_BOXR full rows).
__host__ __device__ __forceinline__ int seg_tile_rows(int mcap, int rr) {
    const int t = mcap > rr ? mcap - rr : 0;
    return (t + SEG_BOXR - 1) / SEG_BOXR * SEG_BOXR;
}
// rr = SEG_REG when every segment has >= SEG_REG + 2 rows, else 0.
__host__ __device__ __forceinline__ int seg_reg_rows(int n_row, int P) {
    return n_row / P >= SEG_REG + 2 ? SEG_REG : 0;
}
__host__ __device__ __forceinline__ size_t seg_smem_bytes(int mcap, int P, bool cyclic,
                                                          bool pascal = true, int rr = 0) {
    const int mt = seg_tile_rows(mcap, rr);
    size_t tiles = (pascal ? 4ull : 3ull) * mt * SEG_S * sizeof(double);
    size_t red = 6ull * SEG_S * sizeof(double);
    size_t rsc = pascal && !seg_rsc_in_b(mt, P, cyclic) ? seg_rsc_bytes(P, cyclic) : 0;
    size_t bars = (size_t)(mt / SEG_BOXR + 1) * sizeof(uint64_t);
    return tiles + red + rsc + bars + 128;  // +128: alignment slack
}

__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// RR: leading rows of each segment held in registers (when every segment has
// at least RR + 2 rows, so rows m - 2 and m - 1 are tile rows).
template <int METHOD, bool CYCLIC, int RR = 0>
__global__ void __launch_bounds__(SEG_S, 5)
seg_f64_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmD,
               const __grid_constant__ CUtensorMap tmX, const SegArgs args) {
    using E = Exact64;
    // every CTA of the cluster reads the same word: all leave together, before
    // any barrier
    if (args.gate != nullptr &&
        ((*static_cast<const volatile unsigned*>(args.gate) != 0u) != (args.gate_run != 0)))
        return;
    extern __shared__ unsigned char smem_raw[];
    double* base = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    constexpr bool STREAM_B = METHOD != SEG_PASCAL;
    static_assert(RR == 0 || RR >= 2, "register rows hold rows 0 and 1");
    constexpr int RRA = RR > 0 ? RR : 1;
    const int mcap = args.mcap;
    const int mt = seg_tile_rows(mcap, RR);  // tile rows
    double* TA = base;
    double* TB = TA + (size_t)mt * SEG_S;  // PaScaL only
    double* TC = TB + (STREAM_B ? 0 : (size_t)mt * SEG_S);
    double* TD = TC + (size_t)mt * SEG_S;
    double* red = TD + (size_t)mt * SEG_S;  // [6][SEG_S]
    double* after_red = red + 6 * SEG_S;
    const bool rsc_in_b = !STREAM_B && seg_rsc_in_b(mt, args.P, CYCLIC);
    double* rsc = rsc_in_b ? TB : after_red;  // reduced-solve scratch (PaScaL)
    const size_t rsc_extra =
        (!STREAM_B && !rsc_in_b) ? seg_rsc_bytes(args.P, CYCLIC) / sizeof(double) : 0;
    uint64_t* bars = reinterpret_cast<uint64_t*>(after_red + rsc_extra);

    cg::cluster_group cluster = cg::this_cluster();
    const int P = args.P;
    const int k = (int)cluster.block_rank();  // segment index
    const int s = threadIdx.x;
    const int g = blockIdx.y;
    const int sys = g * SEG_S + s;
    const bool valid = sys < args.n_sys;
    const size_t ns = (size_t)args.n_sys;

    int r0, m;
    seg_range(args.n_row, P, k, r0, m);
    // rows [0, RR) of the segment live in registers (Filtered), rows [RR, m) in
    // the shared-memory tile (tile row j - RR)
    const int ms = m > RR ? m - RR : 0;
    const int nch = (ms + SEG_BOXR - 1) / SEG_BOXR;

#define T(Z, j) Z[(size_t)((j) - RR) * SEG_S + s]

    // register rows: A, B, C, D straight from HBM (the state then replaces A, C, D)
    double rA[RRA], rB[RRA], rC[RRA], rD[RRA];
    if constexpr (RR > 0) {
#pragma unroll
        for (int u = 0; u < RR; ++u) {
            const bool in = valid && u < m;
            const size_t off = (size_t)(r0 + u) * ns + sys;
            rA[u] = in ? __ldg(args.A + off) : 0.0;
            rB[u] = in ? __ldg(args.B + off) : 1.0;
            rC[u] = in ? __ldg(args.C + off) : 0.0;
            rD[u] = in ? __ldg(args.D + off) : 0.0;
        }
    }

    // ---------------------------------------------------------- stage the tile
    bool ok = true;
    if (args.use_tma) {
        if (s == 0) {
            for (int c = 0; c < nch; ++c) mbar_init(&bars[c], 1);
            fence_mbar_init();
        }
        __syncwarp();
        if (s == 0) {
            const uint32_t bytes = (STREAM_B ? 3u : 4u) * SEG_BOXR * SEG_S * sizeof(double);
            for (int c = 0; c < nch; ++c) {
                mbar_expect_tx(&bars[c], bytes);
                const int y = r0 + RR + c * SEG_BOXR;
                const size_t o = (size_t)c * SEG_BOXR * SEG_S;
                tma_load_2d(TA + o, &tmA, g * SEG_S, y, &bars[c]);
                if (!STREAM_B) tma_load_2d(TB + o, &tmB, g * SEG_S, y, &bars[c]);
                tma_load_2d(TC + o, &tmC, g * SEG_S, y, &bars[c]);
                tma_load_2d(TD + o, &tmD, g * SEG_S, y, &bars[c]);
            }
        }
    } else {
        for (int j = RR; j < m; ++j) {
            size_t off = (size_t)(r0 + j) * ns + sys;
            T(TA, j) = valid ? args.A[off] : 0.0;
            if (!STREAM_B) T(TB, j) = valid ? args.B[off] : 1.0;
            T(TC, j) = valid ? args.C[off] : 0.0;
            T(TD, j) = valid ? args.D[off] : 0.0;
        }
    }
    // B of tile rows [RR + c * SEG_BOXR, RR + (c + 1) * SEG_BOXR) into registers
    // (1 outside the batch or the segment)
    const double* gB = args.B + (size_t)(r0 + RR) * ns + sys;
    auto load_b = [&](int c, double (&bb)[SEG_BOXR]) {
#pragma unroll
        for (int u = 0; u < SEG_BOXR; ++u) {
            const int j = c * SEG_BOXR + u;  // tile row
            bb[u] = (valid && j < ms) ? __ldg(gB + (size_t)j * ns) : 1.0;
        }
    };
    auto chunk_wait = [&](int c) {
        if (args.use_tma && ok) ok = mbar_wait_bounded(&bars[c], 0, args.status);
    };

    // J of this segment (Filtered); v1's interface pass runs the full sweeps.
    int J = m - 1;
    if (METHOD != SEG_PASCAL && !(METHOD == SEG_FILT_V1 && args.mode == SEG_MODE_INTERFACE))
        J = args.J[k];
    const int Jf = (METHOD == SEG_FILT_V2) ? (J < m - 2 ? J : m - 2) : m - 1;  // sweep cutoff
    const int lo = (m - 2) - Jf;

    // ------------------------------------------------------- forward sweep
    double q0, a0, c0, d0, q1, ap, cp, dp;
    double bcur[SEG_BOXR], bnext[SEG_BOXR];  // B of tile chunks c, c + 1 (Filtered)
    if constexpr (RR > 0) {
        q0 = E::rcp(rB[0]);
        a0 = E::mul(rA[0], q0);
        c0 = E::mul(rC[0], q0);
        d0 = E::mul(rD[0], q0);
        q1 = E::rcp(rB[1]);
        ap = E::mul(rA[1], q1);
        cp = E::mul(rC[1], q1);
        dp = E::mul(rD[1], q1);
        rA[0] = a0;
        rC[0] = c0;
        rD[0] = d0;
        rA[1] = ap;
        rC[1] = cp;
        rD[1] = dp;
#pragma unroll
        for (int u = 2; u < RR; ++u) {
            if (u >= m) continue;
            const double a = rA[u];
            const double inv = E::rcp(E::sub(rB[u], E::mul(a, cp)));
            dp = E::mul(inv, E::sub(rD[u], E::mul(a, dp)));
            cp = E::mul(inv, rC[u]);
            rD[u] = dp;
            rC[u] = cp;
            if (METHOD != SEG_FILT_V2 || u <= Jf) {
                ap = E::mul(E::mul(-inv, a), ap);
                rA[u] = ap;
            }
        }
        if (nch > 0) load_b(0, bcur);
        if (nch > 1) load_b(1, bnext);
    } else {
        // rows 0 and 1 are tile rows; B streamed (Filtered) or staged (PaScaL)
        double b0, b1;
        if constexpr (STREAM_B) {
            if (nch > 0) load_b(0, bcur);
            if (nch > 1) load_b(1, bnext);
            b0 = bcur[0];
            b1 = bcur[1];
        }
        chunk_wait(0);
        if constexpr (!STREAM_B) {
            b0 = T(TB, 0);
            b1 = T(TB, 1);
        }
        q0 = E::rcp(b0);
        a0 = E::mul(T(TA, 0), q0);
        c0 = E::mul(T(TC, 0), q0);
        d0 = E::mul(T(TD, 0), q0);
        q1 = E::rcp(b1);
        ap = E::mul(T(TA, 1), q1);
        cp = E::mul(T(TC, 1), q1);
        dp = E::mul(T(TD, 1), q1);
        T(TA, 0) = a0;
        T(TC, 0) = c0;
        T(TD, 0) = d0;
        T(TA, 1) = ap;
        T(TC, 1) = cp;
        T(TD, 1) = dp;
    }
    for (int c = 0; c < nch; ++c) {
        if constexpr (STREAM_B) {
            if (c > 0) {
#pragma unroll
                for (int u = 0; u < SEG_BOXR; ++u) bcur[u] = bnext[u];
                if (c + 1 < nch) load_b(c + 1, bnext);
            }
        }
        if (c > 0 || RR > 0) chunk_wait(c);  // RR == 0: chunk 0 was waited for above
#pragma unroll
        for (int u = 0; u < SEG_BOXR; ++u) {
            const int j = RR + c * SEG_BOXR + u;
            if (j < 2 || j >= m) continue;
            const double a = T(TA, j);
            double bj;
            if constexpr (STREAM_B)
                bj = bcur[u];
            else
                bj = T(TB, j);
            const double inv = E::rcp(E::sub(bj, E::mul(a, cp)));
            dp = E::mul(inv, E::sub(T(TD, j), E::mul(a, dp)));
            cp = E::mul(inv, T(TC, j));
            T(TD, j) = dp;
            T(TC, j) = cp;
            if (METHOD != SEG_FILT_V2 || j <= Jf) {
                ap = E::mul(E::mul(-inv, a), ap);
                T(TA, j) = ap;
            }
        }
    }
    // rows m - 2 and m - 1 are tile rows (m >= RR + 2)
    const double aN = T(TA, m - 1), cN = T(TC, m - 1), dN = T(TD, m - 1);

    // ------------------------------------------------------ backward sweep
    {
        double dn = T(TD, m - 2), an = T(TA, m - 2), cn = T(TC, m - 2);
        // one row of the sweep on (A, C, D) of tile row j
        auto bwd = [&](int j, double& A_, double& C_, double& D_) {
            const double c = C_;
            dn = E::sub(D_, E::mul(c, dn));
            D_ = dn;
            if (METHOD != SEG_FILT_V2 || j < Jf) {
                an = E::sub(A_, E::mul(c, an));
                A_ = an;
            } else {
                an = A_;
            }
            if (METHOD != SEG_FILT_V2 || j > lo) {
                cn = E::mul(c, -cn);
                C_ = cn;
            } else {
                cn = c;
            }
        };
        const int jlo = RR > 1 ? RR : 1;
        for (int j = m - 3; j >= jlo; --j) bwd(j, T(TA, j), T(TC, j), T(TD, j));
        // the register rows: the same steps, indexed directly (no references,
        // which would move the arrays to local memory)
#pragma unroll
        for (int u = RR - 1; u >= 1; --u) {
            if (u > m - 3) continue;
            const double c = rC[u];
            dn = E::sub(rD[u], E::mul(c, dn));
            rD[u] = dn;
            if (METHOD != SEG_FILT_V2 || u < Jf) {
                an = E::sub(rA[u], E::mul(c, an));
                rA[u] = an;
            } else {
                an = rA[u];
            }
            if (METHOD != SEG_FILT_V2 || u > lo) {
                cn = E::mul(c, -cn);
                rC[u] = cn;
            } else {
                cn = c;
            }
        }
    }
    // Row-0 reduction: decouple row 0 from x_1 (pascal_tdma.cpp:173-178,
    // filtered_tdma_kernels.hpp:178-189; Filtered keeps C_0 unreduced).
    {
        double a1, c1, d1;
        if constexpr (RR > 0) {
            a1 = rA[1];
            c1 = rC[1];
            d1 = rD[1];
        } else {
            a1 = T(TA, 1);
            c1 = T(TC, 1);
            d1 = T(TD, 1);
        }
        const double r = E::rcp(E::sub(1.0, E::mul(a1, c0)));
        d0 = E::mul(r, E::sub(d0, E::mul(c0, d1)));
        a0 = E::mul(r, a0);
        if (METHOD == SEG_PASCAL) c0 = E::mul(E::mul(-r, c0), c1);
    }
    red[0 * SEG_S + s] = a0;
    red[1 * SEG_S + s] = c0;
    red[2 * SEG_S + s] = d0;
    red[3 * SEG_S + s] = aN;
    red[4 * SEG_S + s] = cN;
    red[5 * SEG_S + s] = dN;

    // ------------------------------------- exchange through the cluster
    cluster_arrive();
    cluster_wait();

    double x0 = d0, xN = dN;
    if (METHOD == SEG_PASCAL) {
        // Reduced system: rows 2q, 2q+1 = first/last row of segment q, unit
        // diagonal; serial Thomas (tdma_many with B = 1) or its periodic form.
        // All remote rows are gathered first (independent DSMEM loads), then the
        // recurrence runs on local shared memory in place: gc -> c', gd -> d'.
        const int nr = 2 * P;
        double* ga = rsc;                  // [nr][SEG_S]
        double* gc = rsc + nr * SEG_S;
        double* gd = rsc + 2 * nr * SEG_S;
        double* ge = rsc + 3 * nr * SEG_S; // e' (periodic only)
        for (int q = 0; q < P; ++q) {
            const double* rem = cluster.map_shared_rank(red, q);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = 2 * q + h;
                ga[row * SEG_S + s] = rem[(3 * h + 0) * SEG_S + s];
                gc[row * SEG_S + s] = rem[(3 * h + 1) * SEG_S + s];
                gd[row * SEG_S + s] = rem[(3 * h + 2) * SEG_S + s];
            }
        }
#define G(Z, j) Z[(j) * SEG_S + s]
        const double one = E::rcp(1.0);
        if (!CYCLIC) {
            double d = E::mul(G(gd, 0), one), c = E::mul(G(gc, 0), one);
            G(gd, 0) = d;
            G(gc, 0) = c;
            for (int j = 1; j < nr; ++j) {
                const double ra = G(ga, j);
                const double r = E::rcp(E::sub(1.0, E::mul(ra, c)));
                d = E::mul(r, E::sub(G(gd, j), E::mul(ra, d)));
                c = E::mul(r, G(gc, j));
                G(gd, j) = d;
                G(gc, j) = c;
            }
            double x = d;
            for (int j = nr - 2; j >= 2 * k; --j) {
                x = E::sub(G(gd, j), E::mul(G(gc, j), x));
                G(gd, j) = x;
            }
            x0 = G(gd, 2 * k);
            xN = G(gd, 2 * k + 1);
        } else {
            // tdma_cyclic_many on the reduced rows (tdma_local.cpp:108-208), B = 1.
            const int nl = nr - 1;
            const double a_0 = G(ga, 0), c_0 = G(gc, 0), d_0 = G(gd, 0);
            double d = E::mul(G(gd, 1), one), e = E::mul(-G(ga, 1), one), c = E::mul(G(gc, 1), one);
            G(gd, 1) = d;
            G(ge, 1) = e;
            G(gc, 1) = c;
            for (int j = 2; j <= nl; ++j) {
                const double ra = G(ga, j);
                const double e0 = (j == nl) ? -G(gc, j) : 0.0;
                const double r = E::rcp(E::sub(1.0, E::mul(ra, c)));
                d = E::mul(r, E::sub(G(gd, j), E::mul(ra, d)));
                e = E::mul(r, E::sub(e0, E::mul(ra, e)));
                c = E::mul(r, G(gc, j));
                G(gd, j) = d;
                G(ge, j) = e;
                G(gc, j) = c;
            }
            const double d_last = d, e_last = e;
            for (int j = nl - 1; j >= 1; --j) {
                const double cj = G(gc, j);
                d = E::sub(G(gd, j), E::mul(cj, d));
                e = E::sub(G(ge, j), E::mul(cj, e));
                G(gd, j) = d;
                G(ge, j) = e;
            }
            const double xr0 = E::div(E::sub(E::sub(d_0, E::mul(a_0, d_last)), E::mul(c_0, d)),
                                      E::add(E::add(1.0, E::mul(a_0, e_last)), E::mul(c_0, e)));
            auto xr = [&](int j) { return j == 0 ? xr0 : E::add(G(gd, j), E::mul(xr0, G(ge, j))); };
            x0 = xr(2 * k);
            xN = xr(2 * k + 1);
        }
#undef G
    } else {
        int left = k - 1, right = k + 1;
        if (CYCLIC) {
            left = (k + P - 1) % P;
            right = (k + 1) % P;
        }
        if (left >= 0) {
            const double* rem = cluster.map_shared_rank(red, left);
            const double cl = rem[4 * SEG_S + s], dl = rem[5 * SEG_S + s];
            x0 = E::div(E::sub(d0, E::mul(a0, dl)), E::sub(1.0, E::mul(cl, a0)));
        }
        if (right < P) {
            const double* rem = cluster.map_shared_rank(red, right);
            const double ar = rem[0 * SEG_S + s], dr = rem[2 * SEG_S + s];
            xN = E::div(E::sub(dN, E::mul(cN, dr)), E::sub(1.0, E::mul(ar, cN)));
        }
    }
    cluster_arrive();  // this CTA no longer reads its neighbours' shared memory

    if (METHOD == SEG_FILT_V1 && args.mode == SEG_MODE_INTERFACE) {
        // Per-segment max |x0|, |xN| over all systems (non-negative doubles
        // order like their bit patterns).
        unsigned long long b0 = valid ? __double_as_longlong(fabs(x0)) : 0ull;
        unsigned long long bN = valid ? __double_as_longlong(fabs(xN)) : 0ull;
        for (int o = 16; o > 0; o >>= 1) {
            b0 = max(b0, __shfl_xor_sync(0xffffffffu, b0, o));
            bN = max(bN, __shfl_xor_sync(0xffffffffu, bN, o));
        }
        if (s == 0) {
            atomicMax(&args.bnd[2 * k], b0);
            atomicMax(&args.bnd[2 * k + 1], bN);
        }
    } else {
        // ------------------------------------------------ final update
        if constexpr (RR > 0) {
            rD[0] = x0;
        } else {
            T(TD, 0) = x0;
        }
        T(TD, m - 1) = xN;
        if constexpr (METHOD == SEG_PASCAL) {
#pragma unroll
            for (int u = 1; u < RR; ++u)
                if (u < m - 1) rD[u] = E::sub(rD[u], E::add(E::mul(rA[u], x0), E::mul(rC[u], xN)));
            for (int j = RR > 1 ? RR : 1; j < m - 1; ++j)
                T(TD, j) = E::sub(T(TD, j), E::add(E::mul(T(TA, j), x0), E::mul(T(TC, j), xN)));
        } else {
            const int left_end = J < m - 2 ? J : m - 2;
            const int right_beg = (m - 1) - J < 1 ? 1 : (m - 1) - J;
#pragma unroll
            for (int u = 1; u < RR; ++u)
                if (u <= left_end) rD[u] = E::sub(rD[u], E::mul(rA[u], x0));
            for (int j = RR > 1 ? RR : 1; j <= left_end; ++j)
                T(TD, j) = E::sub(T(TD, j), E::mul(T(TA, j), x0));
#pragma unroll
            for (int u = 1; u < RR; ++u)
                if (u >= right_beg && u < m - 1) rD[u] = E::sub(rD[u], E::mul(rC[u], xN));
            for (int j = right_beg > RR ? right_beg : RR; j < m - 1; ++j)
                T(TD, j) = E::sub(T(TD, j), E::mul(T(TC, j), xN));
        }
        bool finite = true;
#pragma unroll
        for (int u = 0; u < RR; ++u)
            if (u < m) finite &= isfinite(rD[u]);
        for (int j = RR; j < m; ++j) finite &= isfinite(T(TD, j));
        if (valid && !finite) raise_status(args.status, ST_NONFINITE);

        // ------------------------------------------------ write x
        if (valid) {
#pragma unroll
            for (int u = 0; u < RR; ++u)
                if (u < m) args.X[(size_t)(r0 + u) * ns + sys] = rD[u];
        }
        const int full = args.use_tma ? ms / SEG_BOXR : 0;  // whole chunks inside the tile
        if (full > 0) {
            fence_async_shared();
            __syncwarp();
            if (s == 0) {
                for (int c = 0; c < full; ++c)
                    tma_store_2d(&tmX, g * SEG_S, r0 + RR + c * SEG_BOXR,
                                 TD + (size_t)c * SEG_BOXR * SEG_S);
                tma_store_commit();
            }
        }
        if (valid)
            for (int j = RR + full * SEG_BOXR; j < m; ++j)
                args.X[(size_t)(r0 + j) * ns + sys] = T(TD, j);
        if (full > 0 && s == 0) tma_store_wait_read();
    }
    if (!ok && args.use_tma) {
        // A chunk wait gave up: give the copies one more bounded chance to land
        // before this CTA's shared memory is released.
        for (int c = 0; c < nch; ++c) mbar_wait_bounded(&bars[c], 0, nullptr, 1u << 16);
    }
    __syncwarp();
    cluster_wait();  // the neighbours are done reading this CTA's shared memory
#undef T
}

}  // namespace btdma
