// Register-tiled segmented solve: the fast exact path (PaScaL, P >= 2).
//
// Every system is cut into NSEG sub-segments of TILE_MT = 16 rows; one thread
// owns one sub-segment of one system and keeps its elimination state in
// registers.  SYS systems are processed together ("a group"); the NSEG
// sub-segments of a group are spread over the CL CTAs of a thread-block cluster
// (CL = 1 for short systems), NSC = NSEG / CL sub-segments per CTA, SYS * NSC
// <= 512 threads.  Persistent clusters walk over the groups:
//
//   1. Forward pass (one row of every local sub-segment per step).  Row k of the
//      CTA's NSC sub-segments of SYS systems arrives in one TMA box of a 3-D view
//      [NSEG][TILE_MT][n_sys] (SYS * 8 bytes wide, 256 B for SYS = 32) through
//      an NST-stage shared-memory ring with one mbarrier per stage; the last warp
//      to finish reading a stage refills it, so the ring stays NST rows ahead of
//      the slowest warp and the next group's rows are in flight while this group
//      finishes.  Each thread runs the modified Thomas elimination of PaScaL
//      (libs/pascal_tdma/cpu/pascal_tdma.cpp:131-170) on its 16 rows:
//          alpha_k x_first + x_k + gamma_k x_{k+1} = delta_k,
//      and, instead of a backward sweep, accumulates the reduced first row in
//      running products: with pi_1 = 1, pi_{k+1} = -gamma_k pi_k,
//          delta''_1 = sum_{k=1}^{M-2} pi_k delta_k, alpha''_1 = sum pi_k alpha_k,
//          gamma''_1 = -pi_{M-1},
//      i.e. the backward recurrence of pascal_tdma.cpp:157-170 at row 1, then the
//      row-0 reduction of pascal_tdma.cpp:173-178.
//   2. Reduced system (the reference's all-to-all + serial Thomas on 2P rows,
//      pascal_tdma.cpp:185-210).  The two reduced rows of every sub-segment are
//      published in shared memory; after a cluster barrier each CTA gathers, over
//      distributed shared memory, the whole reduced system of its SYS/CL systems.
//      One level of cyclic reduction eliminates the first-row unknowns (leaving a
//      tridiagonal system in the last-row unknowns, one row per thread), parallel
//      cyclic reduction solves that in log2(NSEG) barrier steps, and the
//      first-row unknowns follow from their rows.  The results go back to the
//      owning CTAs over distributed shared memory; a second cluster barrier.
//   3. Back substitution from registers: x_k = delta_k - alpha_k x_first -
//      gamma_k x_{k+1}, k = M-2..1, stored coalesced, SYS systems wide.
//
// HBM traffic: A, B, C, D read once (32 B/row), x written once (8 B/row).
// Results equal the serial Thomas solution to rounding (<= 1e-12 relative on
// the tested batches), not bit for bit: the operation order differs from the
// reference's.  Needs n_row = 16 * NSEG, even n_sys and 16-byte aligned arrays
// (TMA); periodic systems need NSEG to be a power of two.
#pragma once

#include <cooperative_groups.h>

#include "btdma_common.cuh"

namespace btdma {

constexpr int TILE_MT = 16;           // rows per sub-segment (per thread)
constexpr int TILE_MAX_THREADS = 512;
constexpr int TILE_MAX_NST = 12;      // ring stages (upper bound)

struct TileArgs {
    double* X;
    int n_sys, n_row;
    int nseg;      // sub-segments per system
    int cl;        // CTAs per cluster (sub-segments split over them)
    int nst;       // ring stages
    int n_groups;  // groups of SYS systems
    unsigned* status;
};

// Shared memory (doubles unless noted), T = SYS * NSC threads, SUB = SYS / CL:
//   ring  NST * 4 * T          TMA stages (A, B, C, D of one row per sub-segment)
//   red   6 * T                this CTA's reduced rows (l0,u0,r0 | l1,u1,r1)
//   gat   6 * (NSEG + 2) * SUB gathered reduced rows, zero guard rows -1, NSEG
//   pcr   6 * (NSEG + 2) * SUB two PCR buffers (a, c, d), guard rows
//   xr    2 * T                x_first / x_last of this CTA's sub-segments
//   bars  NST mbarriers + NST ints
__host__ __device__ __forceinline__ size_t tile_fixed_doubles(int T, int nseg, int sub) {
    return 6ull * T + 6ull * (nseg + 2) * sub + 6ull * (nseg + 2) * sub + 2ull * T;
}
__host__ __device__ __forceinline__ size_t tile_smem_bytes(int T, int nseg, int sub, int nst) {
    return ((size_t)nst * 4 * T + tile_fixed_doubles(T, nseg, sub)) * sizeof(double) +
           (size_t)nst * (sizeof(uint64_t) + sizeof(int)) + 128;
}

__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tile_cluster_sync(int cl) {
    if (cl > 1) {
        asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
        asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    } else {
        __syncthreads();
    }
}

template <int SYS, bool CYCLIC>
__global__ void __launch_bounds__(TILE_MAX_THREADS, 1)
tile_f64_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmD,
                const TileArgs args) {
    namespace cg = cooperative_groups;
    constexpr int M = TILE_MT;
    extern __shared__ unsigned char smem_raw[];
    const int nseg = args.nseg, cl = args.cl, nst = args.nst;
    const int nsc = nseg / cl;   // sub-segments per CTA
    const int T = SYS * nsc;     // == blockDim.x
    const int sub = SYS / cl;    // systems whose reduced system this CTA solves
    const int gs = nseg + 2;     // rows per field in gat / pcr (with guards)

    double* ring = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    double* red = ring + (size_t)nst * 4 * T;
    double* gat = red + 6 * T;
    double* pcr = gat + 6 * gs * sub;
    double* xr = pcr + 6 * gs * sub;
    uint64_t* full = reinterpret_cast<uint64_t*>(xr + 2 * T);
    int* readers = reinterpret_cast<int*>(full + nst);

    const int tid = threadIdx.x;
    const int c = cl > 1 ? (int)cg::this_cluster().block_rank() : 0;
    const int cluster_id = (int)blockIdx.x / cl;
    const int n_clusters = (int)gridDim.x / cl;
    // forward / back-substitution mapping: system s, local sub-segment ql
    const int s = tid % SYS;
    const int ql = tid / SYS;
    // reduced-system mapping: system sp (of this CTA's slice), global sub-segment p
    const int sp = tid % sub;
    const int p = tid / sub;
    const size_t ns = (size_t)args.n_sys;
    const int nwarps = (T + 31) / 32;

    if (tid == 0) {
        for (int i = 0; i < nst; ++i) {
            mbar_init(&full[i], 1);
            readers[i] = 0;
        }
        fence_mbar_init();
    }
    if (tid < sub) {  // zero guard rows of gat and pcr (never written again)
        for (int f = 0; f < 6; ++f) {
            gat[(f * gs + 0) * sub + tid] = 0.0;
            gat[(f * gs + nseg + 1) * sub + tid] = 0.0;
            pcr[(f * gs + 0) * sub + tid] = 0.0;
            pcr[(f * gs + nseg + 1) * sub + tid] = 0.0;
        }
    }
    __syncthreads();
    if (cl > 1) tile_cluster_sync(cl);  // peers' shared memory is live before any DSMEM access

    const int n_my = args.n_groups > cluster_id
                         ? (args.n_groups - cluster_id + n_clusters - 1) / n_clusters
                         : 0;
    const int total = n_my * M;
    const uint32_t stage_bytes = 4u * T * sizeof(double);

    auto issue = [&](int t) {  // one thread
        const int slot = t % nst;
        const int g = cluster_id + (t / M) * n_clusters;
        const int k = t % M;
        double* dst = ring + (size_t)slot * 4 * T;
        mbar_expect_tx(&full[slot], stage_bytes);
        tma_load_3d(dst + 0 * T, &tmA, g * SYS, k, c * nsc, &full[slot]);
        tma_load_3d(dst + 1 * T, &tmB, g * SYS, k, c * nsc, &full[slot]);
        tma_load_3d(dst + 2 * T, &tmC, g * SYS, k, c * nsc, &full[slot]);
        tma_load_3d(dst + 3 * T, &tmD, g * SYS, k, c * nsc, &full[slot]);
    };
    bool ok = true;
    if (tid == 0)
        for (int t = 0; t < nst && t < total; ++t) issue(t);

    // gat / pcr accessors for this thread's reduced-system column (row -1 is
    // the first guard row)
    auto G = [&](int f, int row) -> double& { return gat[(f * gs + row + 1) * sub + sp]; };
    auto PB = [&](int b, int f, int row) -> double& {
        return pcr[((b * 3 + f) * gs + row + 1) * sub + sp];
    };

    bool finite = true;
    int slot = 0;
    uint32_t phase = 0;
    int t = 0;
    for (int it = 0; it < n_my; ++it) {
        const int g = cluster_id + it * n_clusters;
        const int sys = g * SYS + s;
        const bool valid = sys < args.n_sys;

        // ------------------------------------------------------ forward pass
        double al[M], ga[M], de[M];  // rows 1..M-1 used (register resident)
        double ab0 = 0, cb0 = 0, db0 = 0;
        double pi = 1.0, sa = 0.0, sd = 0.0;
#pragma unroll
        for (int k = 0; k < M; ++k) {
            if (ok) ok = mbar_wait_bounded(&full[slot], phase, args.status);
            const double* st = ring + (size_t)slot * 4 * T + tid;
            const double a = st[0], b = st[T], cc = st[2 * T], d = st[3 * T];
            // The last warp to finish reading the slot refills it with stage
            // t + nst: the ring stays nst rows ahead of the slowest warp.
            __syncwarp();
            if ((tid & 31) == 0) {
                __threadfence_block();
                if (atomicAdd(&readers[slot], 1) == nwarps - 1) {
                    readers[slot] = 0;
                    if (ok && t + nst < total) issue(t + nst);
                }
            }
            ++t;
            if (++slot == nst) {
                slot = 0;
                phase ^= 1u;
            }
            if (k == 0) {
                const double ib = rcp_nr(b);
                ab0 = a * ib;
                cb0 = cc * ib;
                db0 = d * ib;
            } else if (k == 1) {
                const double ib = rcp_nr(b);
                al[1] = a * ib;
                ga[1] = cc * ib;
                de[1] = d * ib;
                sa = al[1];
                sd = de[1];
            } else {
                const double inv = rcp_nr(b - a * ga[k - 1]);
                ga[k] = cc * inv;
                de[k] = (d - a * de[k - 1]) * inv;
                al[k] = -a * al[k - 1] * inv;
                if (k <= M - 2) {
                    pi = -ga[k - 1] * pi;
                    sa += pi * al[k];
                    sd += pi * de[k];
                }
            }
        }
        // reduced rows of this sub-segment -> red[f][ql][s]
        {
            const double pi_last = -ga[M - 2] * pi;
            const double r0 = rcp_nr(1.0 - cb0 * sa);
            double* w = red + ql * SYS + s;
            w[0 * T] = r0 * ab0;
            w[1 * T] = r0 * cb0 * pi_last;  // -r c0 gamma''_1, gamma''_1 = -pi_{M-1}
            w[2 * T] = r0 * (db0 - cb0 * sd);
            w[3 * T] = al[M - 1];
            w[4 * T] = ga[M - 1];
            w[5 * T] = de[M - 1];
        }
        tile_cluster_sync(cl);

        // ------------------------------------- gather this CTA's reduced systems
        {
            const int owner = p / nsc;
            const double* src = red + (p % nsc) * SYS + c * sub + sp;
            if (cl > 1 && owner != c) src = cg::this_cluster().map_shared_rank(src, owner);
#pragma unroll
            for (int f = 0; f < 6; ++f) G(f, p) = src[f * T];
        }
        __syncthreads();

        // ------------- one cyclic-reduction level: eliminate the first-row unknowns
        // first row of p:  l0 xL(p-1) + xF(p) + u0 xL(p) = r0
        // last row of p:   l1 xF(p) + xL(p) + u1 xF(p+1) = r1
        const double l0 = G(0, p), u0 = G(1, p), r0 = G(2, p);
        {
            const double l1 = G(3, p), u1 = G(4, p), r1 = G(5, p);
            int pn = p + 1;
            if (CYCLIC && pn == nseg) pn = 0;
            const double l0n = G(0, pn), u0n = G(1, pn), r0n = G(2, pn);
            const double ib = rcp_nr(1.0 - l1 * u0 - u1 * l0n);
            PB(0, 0, p) = -l1 * l0 * ib;
            PB(0, 1, p) = -u1 * u0n * ib;
            PB(0, 2, p) = (r1 - l1 * r0 - u1 * r0n) * ib;
        }
        __syncthreads();

        // ------------------------- PCR on the last-row unknowns (one row/thread)
        int cur = 0;
        double xl;
        if (CYCLIC && nseg == 1) {
            xl = PB(0, 2, 0) * rcp_nr(1.0 + PB(0, 0, 0) + PB(0, 1, 0));
        } else {
            bool solved = false;
            xl = 0.0;
            for (int dl = 1; dl < nseg; dl <<= 1) {
                const bool last_cyclic = CYCLIC && 2 * dl == nseg;
                int im = p - dl, ip = p + dl;
                if (CYCLIC) {
                    im = im < 0 ? im + nseg : im;
                    ip = ip >= nseg ? ip - nseg : ip;
                } else {
                    im = im < -1 ? -1 : im;
                    ip = ip > nseg ? nseg : ip;
                }
                const double li = PB(cur, 0, p), ui = PB(cur, 1, p), ri = PB(cur, 2, p);
                const double lm = PB(cur, 0, im), um = PB(cur, 1, im), rm = PB(cur, 2, im);
                const double lp = PB(cur, 0, ip), up = PB(cur, 1, ip), rp = PB(cur, 2, ip);
                const int nxt = cur ^ 1;
                if (last_cyclic) {
                    // p-dl and p+dl are the same row j: 2x2 system in x_p, x_j
                    const double si = li + ui, sj = lm + um;
                    xl = (ri - si * rm) * rcp_nr(1.0 - si * sj);
                    solved = true;
                } else {
                    const double ib = rcp_nr(1.0 - li * um - ui * lp);
                    PB(nxt, 0, p) = -li * lm * ib;
                    PB(nxt, 1, p) = -ui * up * ib;
                    PB(nxt, 2, p) = (ri - li * rm - ui * rp) * ib;
                }
                __syncthreads();
                cur = nxt;
            }
            if (!solved) xl = PB(cur, 2, p);
        }
        // publish x_last, then recover x_first(p) = r0 - l0 xL(p-1) - u0 xL(p)
        PB(cur ^ 1, 2, p) = xl;
        __syncthreads();
        const int pm = p - 1;
        double xlm;
        if (CYCLIC)
            xlm = PB(cur ^ 1, 2, pm < 0 ? nseg - 1 : pm);
        else
            xlm = pm < 0 ? 0.0 : PB(cur ^ 1, 2, pm);
        const double xf = r0 - l0 * xlm - u0 * xl;
        {
            const int owner = p / nsc;
            double* dst = xr + (p % nsc) * SYS + c * sub + sp;
            if (cl > 1 && owner != c) dst = cg::this_cluster().map_shared_rank(dst, owner);
            dst[0] = xf;
            dst[T] = xl;
        }
        tile_cluster_sync(cl);

        // --------------------------------------------------- back substitution
        const double x_first = xr[ql * SYS + s];
        const double x_last = xr[T + ql * SYS + s];
        if (valid) {
            const int q = c * nsc + ql;
            double* xp = args.X + (size_t)(q * M) * ns + sys;
            xp[(size_t)(M - 1) * ns] = x_last;
            double xn = x_last;
#pragma unroll
            for (int k = M - 2; k >= 1; --k) {
                xn = de[k] - al[k] * x_first - ga[k] * xn;
                finite &= isfinite(xn);
                xp[(size_t)k * ns] = xn;
            }
            xp[0] = x_first;
            finite &= isfinite(x_first) && isfinite(x_last);
        }
    }
    if (!finite) raise_status(args.status, ST_NONFINITE);
    if (!ok && tid == 0) {
        // a wait gave up: give in-flight copies a bounded chance to land before
        // the CTA exits
        for (int i = 0; i < nst; ++i) mbar_wait_bounded(&full[i], 0, nullptr, 1u << 8);
    }
    if (cl > 1) tile_cluster_sync(cl);  // no CTA leaves while peers may touch its memory
}

}  // namespace btdma
