// Register-tiled segmented solve: the fast exact path (PaScaL, P >= 2).
//
// Every system is cut into NSEG sub-segments of TILE_MT = 16 rows; one thread
// owns one sub-segment of one system and keeps its elimination state in
// registers.  SYS systems are processed together ("a group"); the NSEG
// sub-segments of a group are spread over the CL CTAs of a thread-block cluster
// (CL = 1 for short systems), NSC = NSEG / CL sub-segments per CTA, SYS * NSC
// <= 512 threads.  Persistent clusters walk over the groups:
//
//   1. Forward pass (RPS = 2 FP64 or 4 FP32 rows of every local sub-segment per
//      step; 4 FP64 rows when only D is read).
//      Rows k, k+1 of the CTA's NSC sub-segments of SYS systems arrive in one TMA
//      box of a 3-D view [NSEG][TILE_MT][n_sys] (SYS * 8 bytes wide) through an
//      NST-stage shared-memory ring.  Each stage has a "full" mbarrier (TMA
//      transaction count) and an "empty" mbarrier (one arrival per warp); the
//      refill of a stage is issued one row later by a rotating producer warp, so
//      no warp waits for the others on the critical path and the next group's
//      rows are in flight while this group finishes.  Each thread runs the
//      modified Thomas elimination of PaScaL
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
//      distributed shared memory, the reduced systems of its SYS/CL systems, one
//      system per group of W = 2^ceil(log2 NSEG) lanes.  One level of cyclic
//      reduction eliminates the first-row unknowns, parallel cyclic reduction
//      solves the remaining tridiagonal system in the last-row unknowns with warp
//      shuffles (no block barrier), and the first-row unknowns follow.  Systems
//      longer than 512 rows (W > 32) run the same steps through shared memory.
//      The results go back to the owning CTAs; a second cluster barrier.
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
#include "k_reduced.cuh"

namespace btdma {

constexpr int TILE_MT = 16;           // rows per sub-segment (per thread)
// Rows per ring stage: 16 bytes of each array per sub-segment and system, i.e.
// 2 FP64 rows or 4 FP32 rows, so a stage has the same size for both storages;
// 32 bytes (4 FP64 rows) for the D-only ring (na == 1) of the generated-
// coefficient modes, whose per-stage bookkeeping would otherwise cost as much
// as the rows' arithmetic.
__host__ __device__ constexpr int tile_rps(int elem, int na = 4) {
    return (na == 1 ? 32 : 16) / elem;
}
constexpr int TILE_MAX_THREADS = 512;
constexpr int TILE_SH_THREADS = 256;  // CTA size limit of the shared-matrix sweeps
constexpr int TILE_MAX_NST = 8;       // ring stages (upper bound)
constexpr int TILE_MAX_NST_CONST = 16;  // ring stages of D-only (constant-coefficient) rings

// Shared-matrix reduced systems of up to 32 sub-segments: per lane p of the
// shuffle group, the coefficients of every step of reduced_solve_shfl that do
// not depend on the right-hand side (TILE_RED_LANE doubles, lane-major):
//   [0] 1/pivot of the first cyclic-reduction step, [1] l1, [2] u1 (0 where
//   the next sub-segment does not exist), [3] l0, [4] u0, then per PCR level v
//   (distance 2^v, at most 5 levels) [5 + 3v] l, [6 + 3v] u (0 where that
//   neighbour does not exist), [7 + 3v] 1/pivot.
constexpr int TILE_RED_LEVELS = 5;
constexpr int TILE_RED_LANE = 5 + 3 * TILE_RED_LEVELS;
// Offset of the lane table in the factor table of an n_row-row matrix, and
// the whole table's size (rows, sub-segments, lanes).
__host__ __device__ constexpr size_t tile_red_offset(int n_row) {
    return (size_t)n_row * 5 + (size_t)(n_row / 16 + 1) * 6;
}
__host__ __device__ constexpr size_t gen_table_doubles(int n_row) {
    return tile_red_offset(n_row) + 32 * (size_t)TILE_RED_LANE;
}

// TileArgs::mode of the modes that read A, B, C (GEN == 0): bit 0 X +=
// solution (refinement corrections), bit 1 the gate's polarity (run while
// *gate == 0 instead of while *gate != 0), bits 8..15 R > 0: Filtered's
// reduced system with segments of R sub-segments (reduced_solve_filtered)
// instead of the exact one.
constexpr int TILE_MODE_ACCUMULATE = 1;
constexpr int TILE_MODE_GATE_ZERO = 2;
constexpr int TILE_MODE_FILT_SHIFT = 8;

struct TileArgs {
    double* X;
    int n_sys, n_row;
    int nseg;      // sub-segments per system
    int cl;        // CTAs per cluster (sub-segments split over them)
    int nst;       // ring stages
    int n_groups;  // groups of SYS systems
    union {
        struct {  // modes that read A, B, C (GEN == 0)
            int mode;              // TILE_MODE_* bits
            const unsigned* gate;  // non-null: the launch runs only while *gate != 0
                                   // (TILE_MODE_GATE_ZERO: while *gate == 0)
        };
        // Generated-coefficient modes (GEN != 0) may store x through a layout
        // map instead of the plain [n_row][n_sys]: with xblk > 0, row j of
        // system s goes to  X + (s / xblk) * xbs + (s % xblk) * xss + j * xrs
        // (xrs > 0).  The heat step writes its Z sweep in the Y sweep's layout
        // and its X sweep into the ghosted field, without a copy pass.  xrs == 1
        // (a system's rows contiguous) in a shared-matrix sweep of one CTA per
        // group stages the group's x in shared memory and stores every
        // system's rows with coalesced warp stores (the launch adds the tile,
        // tile_tstore_bytes).  (A union with the refinement fields: a larger
        // argument struct made ptxas spill more in every instantiation.)
        struct {
            int xblk, xbs, xss, xrs;
        };
    };
    // Generated-coefficient instantiations read only D:
    //  GEN == 1 (heat sweep): every row -cs x_{j-1} + (1 + 2 cs) x_j - cs x_{j+1},
    //    plus cs on the diagonal of the first and last row when cbound != 0
    //    (the fully implicit Dirichlet wall of the heat ADI step);
    //  GEN == 2 (channel Poisson, wall-normal): row j is
    //    ga[j] x_{j-1} - (ga[j] + gc[j] + glam[s / 2]) x_j + gc[j] x_{j+1},
    //    systems 2m and 2m + 1 being the real and imaginary parts of mode m;
    //    with gpin, row 0 of mode 0 is x_0 = 0 (the pinned mean pressure);
    //  GEN == 3 (channel momentum ADI): row j is
    //    -cs ga[j] x_{j-1} + (1 + cs gb[j]) x_j - cs gc[j] x_{j+1}
    //    (staggered metrics and wall terms folded into the row tables).
    double cs;
    int cbound;
    const double* ga;
    const double* gb;
    const double* gc;
    const double* glam;
    // GEN 1 and 3: every system of the batch has the same matrix, so the
    // elimination of each sub-segment is computed once (tile_table_kernel) into
    // gtab: per row [inv pivot, a * inv, pi, alpha, gamma] (n_row x 5), then
    // per sub-segment [r, r c0, l0, u0, l1, u1] (nseg x 6), then (up to 32
    // sub-segments) the reduced system's lane table at tile_red_offset(n_row);
    // the solve runs the right-hand-side recurrences only
    const double* gtab;
    int gpin;
    unsigned* status;
};

// Reciprocal in the arithmetic of the local sweeps: FP64 with Newton steps, or
// the single-instruction FP32 approximation (the inner solver of refinement).
__device__ __forceinline__ double rcp_tc(double x) { return rcp_nr(x); }
__device__ __forceinline__ float rcp_tc(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__host__ __device__ __forceinline__ int tile_lanes(int nseg) {
    int w = 1;
    while (w < nseg) w <<= 1;
    return w;
}

// Shared memory (doubles unless noted), T = SYS * NSC threads, SUB = SYS / CL,
// RP = SYS + 1 (padded pitch of the exchange buffers):
//   ring  NST * NA * RPS * T      TMA stages (A, B, C, D or D only; RPS rows per sub-segment)
//   red   6 * NSC * RP            this CTA's reduced rows (l0,u0,r0 | l1,u1,r1);
//                                 2 * NSC * RP (r0 | r1) for a shared matrix of
//                                 NSEG <= 32, whose l, u come from the lane table
//   xr    2 * NSC * RP            x_first / x_last of this CTA's sub-segments
//   pcr   6 * (NSEG + 2) * SUB    PCR buffers, only when NSEG > 32
//   tab   tile_tab_doubles(NSC)   shared matrix: this CTA's factor table
//   lane  32 * TILE_RED_LANE      shared matrix, NSEG <= 32: the lane table
//   bars  2 * NST mbarriers
__host__ __device__ __forceinline__ size_t tile_fixed_doubles(int sys, int nsc, int nseg, int sub,
                                                              bool shared_tab = false) {
    if (shared_tab && nseg <= 32) return 4ull * nsc * (sys + 1) + 32ull * TILE_RED_LANE;
    size_t f = 8ull * nsc * (sys + 1);
    if (nseg > 32) f += 6ull * (nseg + 2) * sub;
    return f;
}
// Elements of one ring stage: na arrays of RPS rows of sys systems of nsc
// sub-segments; GEN == 4 (heat Z sweep with the right-hand side fused): a box of
// theta of TILE_HEAT_BOX_I x 3 cells (the 16 systems' columns with their x
// and y neighbours) per row instead of one D value per system.
constexpr int TILE_HEAT_SYS = 16;
constexpr int TILE_HEAT_BOX_I = TILE_HEAT_SYS + 2;
// GEN == 5 (momentum z sweep reading the ghosted field): one row of 18 cells.
// tile_stage_box_elems: what a stage's TMA boxes deliver (its transaction
// count); tile_stage_elems: the distance between stages, rounded up to 128
// bytes, since a tensor copy's shared-memory destination must be 128-byte
// aligned (the 18-cell boxes of GEN 4 / 5 are not, for an odd nsc).
__host__ __device__ __forceinline__ int tile_stage_box_elems(int sys, int nsc, int elem, int na,
                                                             int gen = 0) {
    return gen == 4   ? TILE_HEAT_BOX_I * 3 * tile_rps(elem, na) * nsc
           : gen == 5 ? TILE_HEAT_BOX_I * tile_rps(elem, na) * nsc
                      : na * tile_rps(elem, na) * sys * nsc;
}
__host__ __device__ __forceinline__ int tile_stage_elems(int sys, int nsc, int elem, int na,
                                                         int gen = 0) {
    const int b = tile_stage_box_elems(sys, nsc, elem, na, gen);
    if (gen != 4 && gen != 5) return b;  // rows of SYS systems: whole 128-byte multiples
    const int q = 128 / elem;
    return (b + q - 1) / q * q;
}
// na: arrays per ring stage (4: A, B, C, D; 1: D only).
__host__ __device__ __forceinline__ size_t tile_ring_bytes(int sys, int nsc, int nst, int elem,
                                                           int na = 4, int gen = 0) {
    return (size_t)nst * tile_stage_elems(sys, nsc, elem, na, gen) * elem;
}
// Shared-matrix table slice of one CTA (its nsc sub-segments): per row 5 and
// per sub-segment 6 doubles.
__host__ __device__ __forceinline__ size_t tile_tab_doubles(int nsc) {
    return (size_t)nsc * TILE_MT * 5 + (size_t)nsc * 6;
}
// Row-contiguous stores (xrs == 1): a [sys][rows + 1] tile of x after the
// mbarriers, rows = n_row / PR (a thread owning two sub-segments stages and
// stores the group's two halves in turn); the odd pitch keeps the back
// substitution's writes, 16 systems a warp, on distinct banks.
__host__ __device__ __forceinline__ size_t tile_tstore_bytes(int sys, int rows) {
    return (size_t)sys * (rows + 1) * sizeof(double);
}
__host__ __device__ __forceinline__ size_t tile_smem_bytes(int sys, int nsc, int nseg, int sub,
                                                           int nst, int elem = 8, int na = 4,
                                                           bool shared_tab = false, int gen = 0,
                                                           int tstore_rows = 0) {
    return tile_ring_bytes(sys, nsc, nst, elem, na, gen) +
           (shared_tab ? tile_tab_doubles(nsc) * sizeof(double) : 0) +
           tile_fixed_doubles(sys, nsc, nseg, sub, shared_tab) * sizeof(double) +
           (gen == 4 ? ((size_t)nseg * TILE_MT + 2) * sizeof(double) : 0) +
           2ull * nst * sizeof(uint64_t) + 128 +
           (tstore_rows > 0 ? tile_tstore_bytes(sys, tstore_rows) : 0);
}

__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* smem_dst, const CUtensorMap* map, int x, int y,
                                            int z, int w, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w),
        "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tile_cluster_sync(int cl) {
    if (cl > 1) {
        asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
        asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    } else {
        __syncthreads();
    }
}

// TIN: element type of A, B, C, D in HBM (double, or float).  TC: arithmetic of
// the local sweeps — double (FP32 storage is widened exactly on load), or float
// (the FP32 inner solve of iterative refinement).  The reduced system, the back
// substitution and x are always FP64.
// One CTA per SM in every mode.  (The shared-matrix instantiations, GEN 1 and
// 3, were measured at two CTAs per SM as well: at 64 registers a thread they
// spill and run 1.5x the instructions, which costs more than the second CTA
// hides.)
// PR: sub-segments per thread.  The shared-matrix sweeps keep only delta per
// row, so a thread can own two sub-segments (ql and ql + nsc / 2): half the
// threads per system, two independent recurrences per thread, and CTAs small
// enough that two share an SM and one's reduced solve overlaps the other's
// streaming.
// FILT: the reduced system takes Filtered's 2 x 2 interfaces between segments
// of R = (mode >> TILE_MODE_FILT_SHIFT) sub-segments (a separate
// instantiation: the extra paths would cost the exact kernels registers).
template <int SYS, bool CYCLIC, typename TIN = double, typename TC = double, int GEN = 0,
          int PR = 1, bool FILT = false>
__global__ void __launch_bounds__(TILE_MAX_THREADS, 1)
tile_f64_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmD,
                const TileArgs args) {
    namespace cg = cooperative_groups;
    constexpr int M = TILE_MT;
    constexpr bool CONSTC = GEN != 0;                 // coefficients generated, D only
    // one matrix for all systems (gtab)
    constexpr bool SH = GEN == 1 || GEN == 3 || GEN == 4 || GEN == 5;
    static_assert(GEN != 4 || (SYS == TILE_HEAT_SYS && !CYCLIC), "heat Z sweep: 16 systems");
    static_assert(GEN != 5 || (SYS == TILE_HEAT_SYS && !CYCLIC), "field-box sweep: 16 systems");
    static_assert(PR == 1 || (PR == 2 && SH), "two sub-segments per thread: shared matrix only");
    static_assert(!FILT || GEN == 0, "Filtered interfaces: matrices read from A, B, C");
    constexpr int NA = CONSTC ? 1 : 4;                // arrays per ring stage
    constexpr int RPS = tile_rps((int)sizeof(TIN), NA);  // rows per ring stage
    constexpr int SPG = M / RPS;                         // stages per group
    constexpr int RP = SYS + 1;  // padded pitch of red / xr rows
    extern __shared__ unsigned char smem_raw[];
    const int nseg = args.nseg, cl = args.cl, nst = args.nst;
    const int nsc = nseg / cl;   // sub-segments per CTA
    const int hsc = nsc / PR;    // thread rows: a thread owns sub-segments ql + h * hsc
    const int TS = SYS * nsc;    // columns of a ring stage
    const int T = SYS * hsc;     // == blockDim.x
    const int sub = SYS / cl;    // systems whose reduced system this CTA solves
    const int W = tile_lanes(nseg);
    const bool shuffled = W <= 32;
    const bool rhs_red = SH && shuffled;  // reduced matrix from the lane table
    const int fstride = nsc * RP;  // field stride of red / xr

    TIN* ring = reinterpret_cast<TIN*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const int sstride = tile_stage_elems(SYS, nsc, (int)sizeof(TIN), NA, GEN);  // per stage
    double* red = reinterpret_cast<double*>(ring + (size_t)nst * sstride);
    double* xr = red + (rhs_red ? 2 : 6) * fstride;
    double* pcr = xr + 2 * fstride;  // only when !shuffled
    const int gs = nseg + 2;
    double* tabs = pcr + (shuffled ? 0 : 6 * gs * sub);  // SH: this CTA's factor table
    double* lanes = tabs + (SH ? tile_tab_doubles(nsc) : 0);  // rhs_red: lane table [k][p]
    // GEN == 4: the cos(pi z) table of the rows (ghosts included), read every row
    double* czt = lanes + (rhs_red ? 32 * TILE_RED_LANE : 0);
    uint64_t* full = reinterpret_cast<uint64_t*>(czt + (GEN == 4 ? args.n_row + 2 : 0));
    uint64_t* empty = full + nst;
    // row-contiguous stores through a shared tile (shared-matrix modes, one CTA)
    const bool tstore = SH && args.xblk > 0 && args.xrs == 1 && cl == 1;
    double* xt = reinterpret_cast<double*>(empty + nst);  // [SYS][n_row / PR + 1] when tstore
    const int xtp = args.n_row / PR + 1;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int nwarps = (T + 31) / 32;
    const int c = cl > 1 ? (int)cg::this_cluster().block_rank() : 0;
    const int cluster_id = (int)blockIdx.x / cl;
    const int n_clusters = (int)gridDim.x / cl;
    const int s = tid % SYS;  // forward / back-substitution mapping
    const int ql = tid / SYS;
    // row stride of x: n_sys, or xrs through the layout map of the generated modes
    const size_t ns = (CONSTC && args.xblk > 0) ? (size_t)args.xrs : (size_t)args.n_sys;

    if (tid == 0) {
        for (int i = 0; i < nst; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], nwarps);
        }
        fence_mbar_init();
    }
    if constexpr (SH) {  // rows of this CTA's sub-segments, then their reduced-row factors
        const int c0 = (cl > 1 ? (int)cg::this_cluster().block_rank() : 0) * nsc;
        const double* g0 = args.gtab + (size_t)c0 * M * 5;
        for (int i = threadIdx.x; i < nsc * M * 5; i += blockDim.x) tabs[i] = g0[i];
        const double* g1 = args.gtab + (size_t)args.n_row * 5 + (size_t)c0 * 6;
        for (int i = threadIdx.x; i < nsc * 6; i += blockDim.x) tabs[nsc * M * 5 + i] = g1[i];
        if (rhs_red) {  // lane-major in global memory, field-major here (no bank conflicts)
            const double* g2 = args.gtab + tile_red_offset(args.n_row);
            for (int i = threadIdx.x; i < 32 * TILE_RED_LANE; i += blockDim.x)
                lanes[(i % TILE_RED_LANE) * 32 + i / TILE_RED_LANE] = g2[i];
        }
        if constexpr (GEN == 4)
            for (int i = threadIdx.x; i < args.n_row + 2; i += blockDim.x) czt[i] = args.gc[i];
    }
    if (!shuffled && tid < sub) {  // zero guard rows of the PCR buffers
        for (int f = 0; f < 6; ++f) {
            pcr[(f * gs + 0) * sub + tid] = 0.0;
            pcr[(f * gs + nseg + 1) * sub + tid] = 0.0;
        }
    }
    __syncthreads();
    if (cl > 1) tile_cluster_sync(cl);  // peers' shared memory is live before any DSMEM access

    // a closed gate leaves the CTA without groups (it still runs its setup and
    // exit barriers, so every CTA of a cluster takes the same path)
    const bool gated_off =
        !CONSTC && args.gate != nullptr &&
        ((*static_cast<const volatile unsigned*>(args.gate) == 0u) !=
         ((args.mode & TILE_MODE_GATE_ZERO) != 0));
    // Filtered: lanes per segment of the reduced system
    const int filt_r = FILT ? (args.mode >> TILE_MODE_FILT_SHIFT) & 255 : 0;
    const int n_my = (!gated_off && args.n_groups > cluster_id)
                         ? (args.n_groups - cluster_id + n_clusters - 1) / n_clusters
                         : 0;
    const int total = n_my * SPG;  // ring stages this CTA consumes
    // bytes the TMA boxes of a stage deliver (the 18-cell boxes' stride is padded)
    const uint32_t stage_bytes =
        (GEN == 4 || GEN == 5)
            ? (uint32_t)tile_stage_box_elems(SYS, nsc, (int)sizeof(TIN), NA, GEN) * sizeof(TIN)
            : (uint32_t)sstride * sizeof(TIN);

    auto issue = [&](int t) {  // one thread
        const int slot = t % nst;
        const int g = cluster_id + (t / SPG) * n_clusters;
        const int k0 = (t % SPG) * RPS;
        TIN* dst = ring + (size_t)slot * sstride;
        mbar_expect_tx(&full[slot], stage_bytes);
        if constexpr (GEN == 4) {
            // theta box: x from the system's left neighbour (ghosted index ii0),
            // y = jj - 1 .. jj + 1 (ghosted jj .. jj + 2), RPS rows of every
            // sub-segment (the map's base is plane k = 1)
            const int s0 = g * SYS;
            tma_load_4d(dst, &tmD, s0 % args.xblk, s0 / args.xblk, k0, c * nsc, &full[slot]);
            return;
        }
        if constexpr (GEN == 5) {
            // the field's row (x from the system's left neighbour, ghosted
            // index ii0; y = jj + 1), RPS rows of every sub-segment
            const int s0 = g * SYS;
            tma_load_4d(dst, &tmD, s0 % args.xblk, s0 / args.xblk + 1, k0, c * nsc, &full[slot]);
            return;
        }
        if constexpr (!CONSTC) {
            tma_load_3d(dst + 0 * RPS * T, &tmA, g * SYS, k0, c * nsc, &full[slot]);
            tma_load_3d(dst + 1 * RPS * T, &tmB, g * SYS, k0, c * nsc, &full[slot]);
            tma_load_3d(dst + 2 * RPS * T, &tmC, g * SYS, k0, c * nsc, &full[slot]);
        }
        tma_load_3d(dst + (NA - 1) * RPS * T, &tmD, g * SYS, k0, c * nsc, &full[slot]);
    };
    bool ok = true;
    if (tid == 0)
        for (int t = 0; t < nst && t < total; ++t) issue(t);

    // this thread's element of a stage: array f, row r at st + f*RPS*T + r*SYS
    const int toff = ql * RPS * SYS + s;
    const TIN* st = ring + toff;  // stage t, this thread's column

    double nonfinite = 0.0;  // becomes NaN if any solution entry is NaN or Inf
    int slot = 0;            // ring slot of stage t
    uint32_t phase = 0;      // its phase parity
    int pslot = nst - 1;     // ring slot of stage t - 1
    uint32_t pphase = 1;
    int t = 0;
    int tw = 0;  // t % nwarps
    for (int it = 0; it < n_my; ++it) {
        const int g = cluster_id + it * n_clusters;
        const int sys = g * SYS + s;
        const bool valid = sys < args.n_sys;

        // ------------------------------------------------------ forward pass
        // rows 1..M-1 used (register resident); deP[h]: sub-segment ql + h * hsc
        TC al[M], ga[M], deP[PR][M];
        TC db0P[PR], sdP[PR];
#pragma unroll
        for (int h = 0; h < PR; ++h) db0P[h] = sdP[h] = 0;
        TC(&de)[M] = deP[0];  // the one sub-segment of the PR == 1 modes
        TC& db0 = db0P[0];
        TC& sd = sdP[0];
        double lam = 0.0;  // GEN == 2: this system's diagonal shift
        if constexpr (GEN == 2) lam = valid ? args.glam[sys >> 1] : 0.0;
        TC ab0 = 0, cb0 = 0;
        TC pi = 1, sa = 0;
        if constexpr (GEN == 4) {
            // Heat Z sweep: the right-hand side of every row is computed here
            // from the theta box of the stage (the reference's rhs_kernel and
            // build_lhs_z wall folds, apps/heat_gpu/solve_theta.cu:121-202),
            // with the ghosts computed where read (2 u_BC - theta).  Row k's z
            // neighbours are rows k - 1 and k + 1, so a row is finished one row
            // later; row 0 of the sub-segment takes its lower neighbour from the
            // previous sub-segment's last row in the last stage, row M - 1 its
            // upper one from the next sub-segment's first row in the first.
            const double* hp = args.glam;  // bx, by, dt 3 pi^2, iy, iz
            const int ixg = args.xblk, s0 = g * SYS;
            const int jj = s0 / ixg, ii = s0 % ixg + s;
            const int iy = (int)__ldg(hp + 3), iz = (int)__ldg(hp + 4);
            const double bx = __ldg(hp + 0), by = __ldg(hp + 1), bz = args.cs,
                         srcs = __ldg(hp + 2);
            const double cxi = __ldg(args.ga + ii + 1), cyj = __ldg(args.gb + jj + 1);
            const double diag = 1.0 + (-2.0 * bx) + (-2.0 * by) + (-2.0 * bz);
            const double ubz = -cxi * cyj;
            const double sxy = srcs * cxi * cyj;  // the source term's x, y factor
            // per owned sub-segment: row 0's partial sum, the pending row's
            // partial sum, the previous row's theta, the neighbours' edge rows
            double pp0[PR], pp[PR], pc[PR], tnext[PR], tkm0[PR];
#pragma unroll
            for (int h = 0; h < PR; ++h) pp0[h] = pp[h] = pc[h] = tnext[h] = tkm0[h] = 0.0;
            // the recurrence of the shared-matrix modes on a finished row
            auto feed = [&](int h, int k, double d) {
                const double* tr = tabs + ((ql + h * hsc) * M + k) * 5;
                if (k == 1) {
                    deP[h][1] = d * tr[0];
                    sdP[h] = deP[h][1];
                } else {
                    deP[h][k] = d * tr[0] - tr[1] * deP[h][k - 1];
                    if (k <= M - 2) sdP[h] += tr[2] * deP[h][k];
                }
            };
#pragma unroll
            for (int j = 0; j < SPG; ++j) {
                if (ok) ok = mbar_wait_bounded(&full[slot], phase, args.status);
                // box [sub-segment][row][y][x], x = system + 1 (+-1: x neighbours)
                const double* sb = ring + (size_t)slot * sstride;
                auto at = [&](int qq, int r, int y, int dx) {
                    return sb[((qq * RPS + r) * 3 + y) * TILE_HEAT_BOX_I + s + 1 + dx];
                };
#pragma unroll
                for (int h = 0; h < PR; ++h) {
                    const int qq = ql + h * hsc;  // sub-segment in the CTA
                    const int q = c * nsc + qq;
                    const int kk0 = q * M;
                    if (j == 0 && q + 1 < nseg) tnext[h] = at(qq + 1, 0, 1, 0);
                    if (j == SPG - 1 && q > 0) tkm0[h] = at(qq - 1, RPS - 1, 1, 0);
                    double tc[RPS], tl[RPS], tr_[RPS], ym[RPS], yp[RPS];
#pragma unroll
                    for (int r = 0; r < RPS; ++r) {
                        tc[r] = at(qq, r, 1, 0);
                        tl[r] = at(qq, r, 1, -1);
                        tr_[r] = at(qq, r, 1, 1);
                        ym[r] = at(qq, r, 0, 0);
                        yp[r] = at(qq, r, 2, 0);
                    }
#pragma unroll
                    for (int r = 0; r < RPS; ++r) {
                        const int k = j * RPS + r;
                        const int kk = kk0 + k;
                        const double tt = tc[r];
                        const double czk = czt[kk + 1];
                        const double ux = -cyj * czk, uy = -cxi * czk;  // x, y wall values
                        const double tip = ii + 1 < ixg ? tr_[r] : 2.0 * ux - tt;
                        const double tim = ii > 0 ? tl[r] : 2.0 * ux - tt;
                        const double tjp = jj + 1 < iy ? yp[r] : 2.0 * uy - tt;
                        const double tjm = jj > 0 ? ym[r] : 2.0 * uy - tt;
                        const double src = sxy * czk;
                        double p =
                            (bx * tip + bx * tim) + (by * tjp + by * tjm) + diag * tt + src;
                        if (kk == 0) p += bz * (2.0 * ubz - tt) + bz * ((2.0 * ubz - tt) + tt);
                        if (kk == iz - 1)
                            p += bz * (2.0 * ubz - tt) + bz * ((2.0 * ubz - tt) + tt);
                        if (k >= 1) p += bz * pc[h];  // lower neighbour: the previous row
                        if (k == 1) pp0[h] += bz * tt;  // row 0's upper neighbour
                        if (k >= 2) feed(h, k - 1, pp[h] + bz * tt);
                        if (k == 0)
                            pp0[h] = p;
                        else
                            pp[h] = p;
                        pc[h] = tt;
                    }
                    // PR == 2: one sub-segment's stage values live at a time
                    if constexpr (PR == 2) __syncwarp();
                }
                {  // release the slot (after the arithmetic: measured spill-free)
                    __syncwarp();
                    if (lane == 0) {
                        mbar_arrive(&empty[slot]);
                        if (t >= 1 && warp == tw && t - 1 + nst < total && ok) {
                            ok = mbar_wait_bounded(&empty[pslot], pphase, args.status);
                            if (ok) issue(t - 1 + nst);
                        }
                    }
                    pslot = slot;
                    pphase = phase;
                    ++t;
                    if (++tw == nwarps) tw = 0;
                    if (++slot == nst) {
                        slot = 0;
                        phase ^= 1u;
                    }
                }
            }
            // row M - 1: the next sub-segment's first row above it            // row M - 1: the next sub-segment's first row above it (the top wall's
            // ghost is already in); row 0: the previous sub-segment's last row
            // below it (or the bottom wall's ghost, already in)
#pragma unroll
            for (int h = 0; h < PR; ++h) {
                const int qq = ql + h * hsc;
                const int kk0 = (c * nsc + qq) * M;
                feed(h, M - 1, kk0 + M - 1 == iz - 1 ? pp[h] : pp[h] + bz * tnext[h]);
                db0P[h] = (kk0 == 0 ? pp0[h] : pp0[h] + bz * tkm0[h]) * tabs[(qq * M) * 5];
            }
        } else {
#pragma unroll
            for (int j = 0; j < SPG; ++j) {
                if (ok) ok = mbar_wait_bounded(&full[slot], phase, args.status);
                TIN a2[RPS], b2[RPS], c2[RPS], d2[PR][RPS];  // widened where used
#pragma unroll
                for (int r = 0; r < RPS; ++r) {
                    if constexpr (!CONSTC) {
                        a2[r] = st[0 * RPS * TS + r * SYS];
                        b2[r] = st[1 * RPS * TS + r * SYS];
                        c2[r] = st[2 * RPS * TS + r * SYS];
                    }
#pragma unroll
                    for (int h = 0; h < PR; ++h) {
                        if constexpr (GEN == 5)  // box [sub-segment][row][x], x = system + 1
                            d2[h][r] = ring[(size_t)slot * sstride +
                                            ((ql + h * hsc) * RPS + r) * TILE_HEAT_BOX_I + s + 1];
                        else
                            d2[h][r] = st[(NA - 1) * RPS * TS + h * hsc * RPS * SYS + r * SYS];
                    }
                }
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&empty[slot]);
                    // Rotating producer: one stage later, warp (t % nwarps) refills
                    // the slot of stage t - 1 with stage t - 1 + nst once every warp
                    // has released it.
                    if (t >= 1 && warp == tw && t - 1 + nst < total && ok) {
                        ok = mbar_wait_bounded(&empty[pslot], pphase, args.status);
                        if (ok) issue(t - 1 + nst);
                    }
                }
                pslot = slot;
                pphase = phase;
                ++t;
                if (++tw == nwarps) tw = 0;
                st += sstride;
                if (++slot == nst) {
                    slot = 0;
                    phase ^= 1u;
                    st = ring + toff;
                }
                if constexpr (SH) {  // right-hand side only, factors from gtab
#pragma unroll
                    for (int h = 0; h < PR; ++h)
#pragma unroll
                        for (int r = 0; r < RPS; ++r) {
                            const int k = j * RPS + r;
                            const double* tr = tabs + ((ql + h * hsc) * M + k) * 5;
                            double d = (double)d2[h][r];
                            // GEN == 5 with gpin: row 0 of the system is x = 0
                            // (the w component's first face, k_build_z)
                            if (GEN == 5 && args.gpin != 0 && c * nsc + ql + h * hsc == 0 &&
                                k == 0)
                                d = 0.0;
                            if (k == 0) {
                                db0P[h] = d * tr[0];
                            } else if (k == 1) {
                                deP[h][1] = d * tr[0];
                                sdP[h] = deP[h][1];
                            } else {
                                deP[h][k] = d * tr[0] - tr[1] * deP[h][k - 1];
                                if (k <= M - 2) sdP[h] += tr[2] * deP[h][k];
                            }
                        }
                } else {
#pragma unroll
                    for (int r = 0; r < RPS; ++r) {
                        const int k = j * RPS + r;
                        TC a, b, cc, d = (TC)d2[0][r];
                        if constexpr (GEN == 2) {
                            const int kg = (c * nsc + ql) * M + k;  // row of the system
                            const double ta = args.ga[kg], tc = args.gc[kg];
                            a = (TC)ta;
                            cc = (TC)tc;
                            b = (TC)(-(ta + tc) - lam);
                            if (args.gpin != 0 && kg == 0 && (sys >> 1) == 0) {
                                a = 0;
                                b = 1;
                                cc = 0;
                                d = 0;
                            }
                        } else {
                            a = (TC)a2[r];
                            b = (TC)b2[r];
                            cc = (TC)c2[r];
                        }
                        if (k == 0) {
                            const TC ib = rcp_tc(b);
                            ab0 = a * ib;
                            cb0 = cc * ib;
                            db0 = d * ib;
                        } else if (k == 1) {
                            const TC ib = rcp_tc(b);
                            al[1] = a * ib;
                            ga[1] = cc * ib;
                            de[1] = d * ib;
                            sa = al[1];
                            sd = de[1];
                        } else {
                            const TC inv = rcp_tc(b - a * ga[k - 1]);
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
                }
            }
        }
        // reduced rows of this sub-segment -> red[f][ql][s]
        if constexpr (SH) {
#pragma unroll
            for (int h = 0; h < PR; ++h) {
                const int qq = ql + h * hsc;
                const double* sb = tabs + nsc * M * 5 + qq * 6;
                double* w = red + qq * RP + s;
                if (rhs_red) {  // r0 | r1 only
                    w[0] = sb[0] * (double)db0P[h] - sb[1] * (double)sdP[h];
                    w[fstride] = (double)deP[h][M - 1];
                } else {
                    w[2 * fstride] = sb[0] * (double)db0P[h] - sb[1] * (double)sdP[h];
                    w[5 * fstride] = (double)deP[h][M - 1];
                    w[0 * fstride] = sb[2];
                    w[1 * fstride] = sb[3];
                    w[3 * fstride] = sb[4];
                    w[4 * fstride] = sb[5];
                }
            }
        } else {
            const TC pi_last = -ga[M - 2] * pi;
            const TC r0 = rcp_tc(TC(1) - cb0 * sa);
            double* w = red + ql * RP + s;
            w[0 * fstride] = (double)(r0 * ab0);
            w[1 * fstride] = (double)(r0 * cb0 * pi_last);  // -r c0 gamma''_1, gamma''_1 = -pi_{M-1}
            w[2 * fstride] = (double)(r0 * (db0 - cb0 * sd));
            w[3 * fstride] = (double)al[M - 1];
            w[4 * fstride] = (double)ga[M - 1];
            w[5 * fstride] = (double)de[M - 1];
        }
        tile_cluster_sync(cl);

        // ------------------------------------------------------ reduced system
        // Row notation for sub-segment p (of one system):
        //   first: l0 xL(p-1) + xF(p) + u0 xL(p) = r0
        //   last:  l1 xF(p) + xL(p) + u1 xF(p+1) = r1
        // One cyclic-reduction level leaves  a xL(p-1) + xL(p) + c xL(p+1) = d.
        if (shuffled) {
            const int per_pass = T / W;  // systems per pass
            const int p = tid % W;
            for (int base = 0; base < sub; base += per_pass) {
                const int sp = base + tid / W;
                const bool act = sp < sub && p < nseg;
                double l0 = 0, u0 = 0, r0 = 0, l1 = 0, u1 = 0, r1 = 0;
                if (act) {
                    const int owner = p / nsc;
                    const double* src = red + (p % nsc) * RP + c * sub + sp;
                    if (cl > 1 && owner != c) src = cg::this_cluster().map_shared_rank(src, owner);
                    r0 = src[(SH ? 0 : 2) * fstride];
                    r1 = src[(SH ? 1 : 5) * fstride];
                    if constexpr (!SH) {
                        l0 = src[0 * fstride];
                        u0 = src[1 * fstride];
                        l1 = src[3 * fstride];
                        u1 = src[4 * fstride];
                    }
                }
                double xf, xl;
                if constexpr (SH)
                    reduced_solve_rhs<CYCLIC>(r0, r1, p, nseg, W, lanes + p, 32, xf, xl);
                else if constexpr (FILT)
                    reduced_solve_filtered<CYCLIC>(l0, u0, r0, l1, u1, r1, p, nseg, W, filt_r,
                                                   act, xf, xl);
                else
                    reduced_solve_shfl<CYCLIC>(l0, u0, r0, l1, u1, r1, p, nseg, W, act, xf, xl);
                if (act) {
                    const int owner = p / nsc;
                    double* dst = xr + (p % nsc) * RP + c * sub + sp;
                    if (cl > 1 && owner != c) dst = cg::this_cluster().map_shared_rank(dst, owner);
                    dst[0] = xf;
                    dst[fstride] = xl;
                }
            }
        } else {
            // NSEG > 32: the same steps through shared memory, one row per thread.
            const int sp = tid % sub;
            const int p = tid / sub;
            auto PB = [&](int b, int f, int row) -> double& {
                return pcr[((b * 3 + f) * gs + row + 1) * sub + sp];
            };
            const int owner = p / nsc;
            const double* src = red + (p % nsc) * RP + c * sub + sp;
            if (cl > 1 && owner != c) src = cg::this_cluster().map_shared_rank(src, owner);
            const double l0 = src[0 * fstride], u0 = src[1 * fstride], r0 = src[2 * fstride];
            const double l1 = src[3 * fstride], u1 = src[4 * fstride], r1 = src[5 * fstride];
            // publish the first rows for the neighbour (field 0..2 of buffer 1)
            PB(1, 0, p) = l0;
            PB(1, 1, p) = u0;
            PB(1, 2, p) = r0;
            __syncthreads();
            int pn = p + 1;
            if (CYCLIC && pn == nseg) pn = 0;
            const double l0n = PB(1, 0, pn), u0n = PB(1, 1, pn), r0n = PB(1, 2, pn);
            {
                const double ib = rcp_nr(1.0 - l1 * u0 - u1 * l0n);
                PB(0, 0, p) = -l1 * l0 * ib;
                PB(0, 1, p) = -u1 * u0n * ib;
                PB(0, 2, p) = (r1 - l1 * r0 - u1 * r0n) * ib;
            }
            __syncthreads();
            int cur = 0;
            double xl = 0.0;
            bool solved = false;
            for (int dl = 1; dl < nseg; dl <<= 1) {
                int im = p - dl, ip = p + dl;
                if (CYCLIC) {
                    im = im < 0 ? im + nseg : im;
                    ip = ip >= nseg ? ip - nseg : ip;
                } else {
                    im = im < -1 ? -1 : im;
                    ip = ip > nseg ? nseg : ip;
                }
                double li = PB(cur, 0, p), ui = PB(cur, 1, p), ri = PB(cur, 2, p);
                const double lm = PB(cur, 0, im), um = PB(cur, 1, im), rm = PB(cur, 2, im);
                const double lp = PB(cur, 0, ip), up = PB(cur, 1, ip), rp = PB(cur, 2, ip);
                const int nxt = cur ^ 1;
                if (CYCLIC && 2 * dl == nseg) {
                    const double si = li + ui, sj = lm + um;
                    xl = (ri - si * rm) * rcp_nr(1.0 - si * sj);
                    solved = true;
                } else {
                    pcr_step(li, ui, ri, lm, um, rm, lp, up, rp);
                    PB(nxt, 0, p) = li;
                    PB(nxt, 1, p) = ui;
                    PB(nxt, 2, p) = ri;
                }
                __syncthreads();
                cur = nxt;
            }
            if (!solved) xl = PB(cur, 2, p);
            PB(cur ^ 1, 2, p) = xl;
            __syncthreads();
            const int pm = p - 1;
            double xlm;
            if (CYCLIC)
                xlm = PB(cur ^ 1, 2, pm < 0 ? nseg - 1 : pm);
            else
                xlm = pm < 0 ? 0.0 : PB(cur ^ 1, 2, pm);
            const double xf = r0 - l0 * xlm - u0 * xl;
            double* dst = xr + (p % nsc) * RP + c * sub + sp;
            if (cl > 1 && owner != c) dst = cg::this_cluster().map_shared_rank(dst, owner);
            dst[0] = xf;
            dst[fstride] = xl;
        }
        tile_cluster_sync(cl);

        // --------------------------------------------------- back substitution
#pragma unroll
        for (int h = 0; h < PR; ++h) {
            const int qq = ql + h * hsc;  // sub-segment in the CTA
            const double x_first = xr[qq * RP + s];
            const double x_last = xr[fstride + qq * RP + s];
            if (valid) {
                const int q = c * nsc + qq;
                double* xp = args.X + (size_t)(q * M + M - 1) * ns + sys;  // row M-1
                if constexpr (CONSTC) {
                    if (tstore)  // staged, rows contiguous (relative to this half's first row)
                        xp = xt + (size_t)s * xtp + ql * M + M - 1;
                    else if (args.xblk > 0)
                        xp = args.X + (ptrdiff_t)(sys / args.xblk) * (ptrdiff_t)args.xbs +
                             (ptrdiff_t)(sys % args.xblk) * (ptrdiff_t)args.xss +
                             (size_t)(q * M + M - 1) * ns;
                }
                // corrections are accumulated only by the FP32 inner solve of
                // refinement (the FP64-arithmetic instantiations keep the plain
                // store); the old x of all M rows is loaded before any store
                double xo[M] = {};
                bool acc = false;
                if constexpr (sizeof(TC) == 4) {
                    acc = (args.mode & TILE_MODE_ACCUMULATE) != 0;
                    if (acc) {
#pragma unroll
                        for (int k = 0; k < M; ++k) xo[k] = xp[-(ptrdiff_t)(M - 1 - k) * (ptrdiff_t)ns];
                    }
                }
                *xp = acc ? xo[M - 1] + x_last : x_last;
                double xn = x_last;
#pragma unroll
                for (int k = M - 2; k >= 1; --k) {
                    xp -= ns;
                    if constexpr (SH) {
                        const double* tr = tabs + (qq * M + k) * 5;
                        xn = (double)deP[h][k] - tr[3] * x_first - tr[4] * xn;
                    } else {
                        xn = (double)de[k] - (double)al[k] * x_first - (double)ga[k] * xn;
                    }
                    nonfinite = fma(xn, 0.0, nonfinite);
                    *xp = acc ? xo[k] + xn : xn;
                }
                xp -= ns;
                *xp = acc ? xo[0] + x_first : x_first;
                nonfinite = fma(x_first, 0.0, fma(x_last, 0.0, nonfinite));
            }
            if (tstore) {
                // this half's x from the tile, each system's rows by one warp
                // with coalesced stores; the tile is written again after the
                // barrier below, or after the next group's two barriers
                const int r0 = h * hsc * M, nr = hsc * M;
                __syncthreads();
                for (int ss = warp; ss < SYS; ss += nwarps) {
                    const int sg = g * SYS + ss;
                    if (sg >= args.n_sys) break;
                    double* dst = args.X + (ptrdiff_t)(sg / args.xblk) * (ptrdiff_t)args.xbs +
                                  (ptrdiff_t)(sg % args.xblk) * (ptrdiff_t)args.xss + r0;
                    const double* src = xt + (size_t)ss * xtp;
                    for (int r = lane; r < nr; r += 32) dst[r] = src[r];
                }
                if (h + 1 < PR) __syncthreads();
            }
        }
    }
    if (nonfinite != 0.0) raise_status(args.status, ST_NONFINITE);  // NaN != 0
    if (!ok && tid == 0) {
        // a wait gave up: give in-flight copies a bounded chance to land before
        // the CTA exits
        for (int i = 0; i < nst; ++i) mbar_wait_bounded(&full[i], 0, nullptr, 1u << 8);
    }
    if (cl > 1) tile_cluster_sync(cl);  // no CTA leaves while peers may touch its memory
}

// Coefficients (a, b, c) of row k of sub-segment q for the shared-matrix modes,
// as the solve generates them.
template <int GEN>
__device__ __forceinline__ void tile_gen_row(const TileArgs& args, int q, int k, double& a,
                                             double& b, double& c) {
    if constexpr (GEN == 1) {
        const bool wall =
            args.cbound != 0 && ((q == 0 && k == 0) || (q == args.nseg - 1 && k == TILE_MT - 1));
        a = -args.cs;
        c = -args.cs;
        b = 1.0 + 2.0 * args.cs + (wall ? args.cs : 0.0);
    } else {
        const int kg = q * TILE_MT + k;
        a = -args.cs * args.ga[kg];
        c = -args.cs * args.gc[kg];
        b = 1.0 + args.cs * args.gb[kg];
    }
}

// The elimination of every sub-segment of the shared matrix (the steps of the
// tiled kernel's forward pass and reduced-row formation without the right-hand
// side): one thread per sub-segment; then, for up to 32 sub-segments, warp 0
// runs the matrix steps of the reduced system into the lane table.
template <int GEN, bool CYCLIC>
__global__ void tile_table_kernel(const TileArgs args, double* __restrict__ tab) {
    constexpr int M = TILE_MT;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < args.nseg) {
        double* sub = tab + (size_t)args.n_row * 5 + (size_t)q * 6;
        double ab0 = 0, cb0 = 0, sa = 0, pi = 1.0, alp = 0, gap = 0, gm2 = 0;
        double ra[M], rb[M], rc[M];  // every row's coefficients before the recurrence
#pragma unroll
        for (int k = 0; k < M; ++k) tile_gen_row<GEN>(args, q, k, ra[k], rb[k], rc[k]);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            const double a = ra[k], b = rb[k], c = rc[k];
            double* tr = tab + (size_t)(q * M + k) * 5;
            if (k == 0) {
                const double ib = rcp_nr(b);
                ab0 = a * ib;
                cb0 = c * ib;
                tr[0] = ib;
                tr[1] = tr[2] = tr[3] = tr[4] = 0.0;
                continue;
            }
            double al, ga, inv;
            if (k == 1) {
                inv = rcp_nr(b);
                al = a * inv;
                ga = c * inv;
                sa = al;
                tr[1] = 0.0;
                tr[2] = 1.0;
            } else {
                inv = rcp_nr(b - a * gap);
                ga = c * inv;
                al = -a * alp * inv;
                tr[1] = a * inv;
                if (k <= M - 2) {
                    pi = -gap * pi;
                    sa += pi * al;
                }
                tr[2] = pi;
            }
            tr[0] = inv;
            tr[3] = al;
            tr[4] = ga;
            if (k == M - 2) gm2 = ga;
            alp = al;
            gap = ga;
        }
        const double pi_last = -gm2 * pi;
        const double rr = rcp_nr(1.0 - cb0 * sa);
        sub[0] = rr;
        sub[1] = rr * cb0;
        sub[2] = rr * ab0;
        sub[3] = rr * cb0 * pi_last;
        sub[4] = alp;
        sub[5] = gap;
    }
    const int nseg = args.nseg;
    if (nseg > 32 || blockIdx.x != 0) return;
    __syncthreads();  // one CTA holds every sub-segment when nseg <= 32
    if (threadIdx.x >= 32) return;
    const int W = tile_lanes(nseg);
    const int p = threadIdx.x & (W - 1);
    const bool act = p < nseg;
    const double* sb = tab + (size_t)args.n_row * 5 + (size_t)p * 6;
    const double l0 = act ? sb[2] : 0.0, u0 = act ? sb[3] : 0.0;
    const double l1 = act ? sb[4] : 0.0, u1 = act ? sb[5] : 0.0;
    double* lt = (int)threadIdx.x < W
                     ? tab + tile_red_offset(args.n_row) + (size_t)p * TILE_RED_LANE
                     : nullptr;
    reduced_lane_table<CYCLIC>(l0, u0, l1, u1, p, nseg, W, act, lt);
}

}  // namespace btdma
