// C ABI of the batched tridiagonal library (declared in include/btdma.h).
//
// One translation unit: the kernels are header-only (k_*.cuh) and instantiated
// here.  The handle owns every device buffer a solve needs (allocated once in
// btdma_create), so solves allocate nothing and can be captured in CUDA graphs.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "btdma_common.cuh"
#include "k_filtered_j.cuh"
#include "k_heat.cuh"
#include "k_momentum.cuh"
#include "k_ragged.cuh"
#include "k_refine.cuh"
#include "k_segment.cuh"
#include "k_thomas.cuh"
#include "k_tile.cuh"

using namespace btdma;

struct btdma_handle {
    int method, P, precision, flags;
    int n_sys_cap, n_row_cap;
    double eps_constant;
    double* rho_row = nullptr;               // [n_row_cap] per-row spectral bound
    int* J = nullptr;                        // [P]
    unsigned long long* work = nullptr;      // [2P] J accumulators (kept zero between solves)
    unsigned* status = nullptr;              // device status word
    double* scratch = nullptr;               // P == 1: c' and e' [2][n_row_cap * n_sys_cap]
    cudaStream_t last_stream = nullptr;
    // FP32_REFINE: residual [n_row_cap * n_sys_cap] (FP32), per-system sweep
    // counts [n_sys_cap], open-system counters [BTDMA_REFINE_MAX_SWEEPS + 1]
    float* resid = nullptr;
    unsigned char* iters = nullptr;
    unsigned* open = nullptr;
    int max_sweeps = 3;
    double eta_tol = 8.0 * 0x1p-53;
    int last_n_sys = 0;
    bool last_refined = false;
    // ragged batches: the plan of the most recent row-offset layout
    struct RagBucket {
        int cyc, first, count, nmin, nmax;
        int cta;    // 1: one CTA of P threads per system, 0: P lanes of a warp per system
        int staged; // CTA kind: system staged through shared memory (autotuner's choice)
        int P, warps, mcap;
        float best_ms;
    };
    std::vector<long long> rag_off;        // host copy of the offsets of the plan
    std::vector<unsigned char> rag_per;    // host copy of the periodic flags
    std::vector<RagBucket> rag_buckets;
    std::vector<int> rag_order;            // system ids, bucket by bucket
    long long* rag_d_off = nullptr;        // device offsets [n_sys + 1]
    int* rag_d_list = nullptr;             // device copy of rag_order
    int4* rag_d_tasks = nullptr;           // task tables [2 * n_sys]
    int4* rag_d_probe = nullptr;           // task table of one bucket being tuned [n_sys]
    // launches of a solve: warp-kind tasks (one launch), CTA-kind tasks per P
    struct RagLaunch {
        int cta, P, first, count, mcap, staged;
    };
    std::vector<RagLaunch> rag_launches;
    static constexpr int RAG_STREAMS = 4;
    cudaStream_t rag_side[RAG_STREAMS] = {};
    cudaEvent_t rag_fork = nullptr, rag_join[RAG_STREAMS] = {};
};

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(BTDMA_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                              \
    } while (0)

// ------------------------------------------------------------ tensor maps
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// [n_row x n_sys] FP64 array, boxes of SEG_BOXR rows x SEG_S systems.
bool make_map(CUtensorMap* map, const void* ptr, int n_sys, int n_row) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)n_sys, (cuuint64_t)n_row};
    cuuint64_t strides[1] = {(cuuint64_t)n_sys * sizeof(double)};
    cuuint32_t box[2] = {(cuuint32_t)SEG_S, (cuuint32_t)SEG_BOXR};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(ptr), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool tma_ok(const void* p, int n_sys) {
    return ((reinterpret_cast<uintptr_t>(p) & 15) == 0) && (n_sys % 2 == 0);
}

int auto_segments(int n_row) {
    // ~64 rows per segment, at least 3, at most the cluster limit.
    if (n_row < 6) return 1;
    int P = (n_row + 63) / 64;
    P = std::max(2, std::min(P, SEG_MAX_P));
    while (P > 1 && n_row / P < 3) --P;
    return P;
}

int seg_mcap(int n_row, int P) {
    int mmax = (n_row + P - 1) / P;
    return (mmax + SEG_BOXR - 1) / SEG_BOXR * SEG_BOXR;
}

int max_smem_optin() {
    static int v = -1;
    if (v < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
            v = 48 * 1024;
    }
    return v;
}

template <int METHOD, bool CYCLIC>
int launch_seg(const CUtensorMap* maps, const SegArgs& a, int groups, cudaStream_t st) {
    auto kern = seg_f64_kernel<METHOD, CYCLIC>;
    static bool attr_done = false;
    if (!attr_done) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                max_smem_optin()));
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        attr_done = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(a.P, groups, 1);
    cfg.blockDim = dim3(SEG_S, 1, 1);
    cfg.dynamicSmemBytes = seg_smem_bytes(a.mcap, a.P, CYCLIC);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.P;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, kern, maps[0], maps[1], maps[2], maps[3], maps[4], a));
    return BTDMA_OK;
}

// 3-D view [nseg][TILE_MT][n_sys] of an [n_row x n_sys] FP64 array; boxes of
// tile_rps(elem) rows of `nsc` consecutive sub-segments for `sys` systems.
bool make_tile_map(CUtensorMap* map, const void* ptr, int n_sys, int nseg, int sys, int nsc,
                   int elem = 8) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {(cuuint64_t)n_sys, (cuuint64_t)TILE_MT, (cuuint64_t)nseg};
    cuuint64_t strides[2] = {(cuuint64_t)n_sys * elem, (cuuint64_t)n_sys * TILE_MT * elem};
    cuuint32_t box[3] = {(cuuint32_t)sys, (cuuint32_t)tile_rps(elem), (cuuint32_t)nsc};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                    3, const_cast<void*>(ptr), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

int num_sms() {
    static int v = -1;
    if (v < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) v = 1;
    }
    return v;
}

// Shape plan of the tiled kernel: systems per group, CTAs per cluster, ring stages.
struct TilePlan {
    int sys = 0, cl = 0, nst = 0, nseg = 0;
};

int max_smem_per_sm() {
    static int v = -1;
    if (v < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) !=
            cudaSuccess)
            v = 0;
    }
    return v;
}

// na: arrays per ring stage (4, or 1 for the constant-coefficient D-only ring).
// sh: shared-matrix sweep (factor table in shared memory, two CTAs per SM).
TilePlan tile_plan(int n_row, bool cyclic, int elem = 8, int na = 4, bool sh = false) {
    TilePlan pl;
    if (n_row % TILE_MT != 0) return pl;
    const int nseg = n_row / TILE_MT;
    if (cyclic && (nseg & (nseg - 1)) != 0) return pl;  // periodic PCR needs 2^k rows
    int sys, cl = 0;
    if (nseg <= 4) {
        sys = 128;
        cl = 1;
    } else if (nseg <= 8) {
        sys = 64;
        cl = 1;
    } else if (nseg <= 16) {
        sys = 32;
        cl = 1;
    } else {
        // One CTA up to 32 sub-segments (a 2-CTA cluster with 256-byte boxes
        // measured slower than one CTA with 128-byte boxes); longer systems split
        // over the smallest cluster that keeps <= 32 sub-segments per CTA.
        sys = 16;
        for (int c = 1; c <= 16; c <<= 1)
            if (nseg % c == 0 && nseg / c <= 32) {
                cl = c;
                break;
            }
        if (cl == 0) return pl;
    }
    int nst = na == 4 ? TILE_MAX_NST : TILE_MAX_NST_CONST;
    // two CTAs per SM for shared-matrix sweeps: half an SM's shared memory each
    // (less 1 KB the runtime reserves per CTA)
    const size_t cap = sh && cl == 1 ? (size_t)max_smem_per_sm() / 2 - 1024 : (size_t)max_smem_optin();
    while (nst >= 3 &&
           tile_smem_bytes(sys, nseg / cl, nseg, sys / cl, nst, elem, na, sh) > cap)
        --nst;
    if (nst < 3) return pl;
    pl.sys = sys;
    pl.cl = cl;
    pl.nst = nst;
    pl.nseg = nseg;
    return pl;
}

template <int SYS, bool CYCLIC, typename TIN = double, typename TC = double, int GEN = 0>
int launch_tile_sys(const CUtensorMap* maps, const TileArgs& a, cudaStream_t st) {
    auto kern = tile_f64_kernel<SYS, CYCLIC, TIN, TC, GEN>;
    static bool attr_done = false;
    if (!attr_done) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                max_smem_optin()));
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        attr_done = true;
    }
    const int threads = SYS * a.nseg / a.cl;
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(threads, 1, 1);
    constexpr bool SHT = GEN == 1 || GEN == 3;
    cfg.dynamicSmemBytes = tile_smem_bytes(SYS, a.nseg / a.cl, a.nseg, SYS / a.cl, a.nst,
                                           (int)sizeof(TIN), GEN ? 1 : 4, SHT);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = num_sms();
    if (SHT && a.cl == 1) {  // built for two CTAs per SM
        int nb = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads,
                                                         cfg.dynamicSmemBytes));
        clusters = num_sms() * std::max(1, nb);
    }
    if (a.cl > 1) {
        cfg.gridDim = dim3(a.cl * num_sms(), 1, 1);
        int nc = 0;
        CK(cudaOccupancyMaxActiveClusters(&nc, kern, &cfg));
        if (nc <= 0) return fail(BTDMA_ERR_UNSUPPORTED, "no cluster of %d CTAs fits", a.cl);
        clusters = nc;
    }
    clusters = std::min(clusters, a.n_groups);
    cfg.gridDim = dim3(clusters * a.cl, 1, 1);
    TileArgs aa = a;
    CK(cudaLaunchKernelEx(&cfg, kern, maps[0], maps[1], maps[2], maps[3], aa));
    return BTDMA_OK;
}

template <typename TIN, typename TC>
int launch_tile_plan(const TilePlan& pl, const CUtensorMap* maps, const TileArgs& a, bool cyclic,
                     cudaStream_t st) {
    switch (pl.sys * 2 + (cyclic ? 1 : 0)) {
        case 256: return launch_tile_sys<128, false, TIN, TC>(maps, a, st);
        case 257: return launch_tile_sys<128, true, TIN, TC>(maps, a, st);
        case 128: return launch_tile_sys<64, false, TIN, TC>(maps, a, st);
        case 129: return launch_tile_sys<64, true, TIN, TC>(maps, a, st);
        case 64: return launch_tile_sys<32, false, TIN, TC>(maps, a, st);
        case 65: return launch_tile_sys<32, true, TIN, TC>(maps, a, st);
        case 33: return launch_tile_sys<16, true, TIN, TC>(maps, a, st);
        default: return launch_tile_sys<16, false, TIN, TC>(maps, a, st);
    }
}

bool tma_ok_elem(const void* p, int n_sys, int elem) {
    return ((reinterpret_cast<uintptr_t>(p) & 15) == 0) && ((size_t)n_sys * elem) % 16 == 0;
}

// Returns 1 when the tiled kernel was launched, 0 when the shape needs the
// cluster-per-segment kernel, < 0 on error.
// TC: arithmetic of the local sweeps; accumulate: X += solution; gate: the
// kernel does nothing while *gate == 0.
template <typename TIN, typename TC = double>
int try_tile(const TIN* A, const TIN* B, const TIN* C, const TIN* D, double* X, int n_sys,
             int n_row, bool cyclic, unsigned* status, cudaStream_t st, bool accumulate = false,
             const unsigned* gate = nullptr) {
    const int elem = (int)sizeof(TIN);
    const TilePlan pl = tile_plan(n_row, cyclic, elem);
    if (pl.sys == 0) return 0;
    if (!(tma_ok_elem(A, n_sys, elem) && tma_ok_elem(B, n_sys, elem) &&
          tma_ok_elem(C, n_sys, elem) && tma_ok_elem(D, n_sys, elem)))
        return 0;
    const int nsc = pl.nseg / pl.cl;
    CUtensorMap maps[4];
    if (!(make_tile_map(&maps[0], A, n_sys, pl.nseg, pl.sys, nsc, elem) &&
          make_tile_map(&maps[1], B, n_sys, pl.nseg, pl.sys, nsc, elem) &&
          make_tile_map(&maps[2], C, n_sys, pl.nseg, pl.sys, nsc, elem) &&
          make_tile_map(&maps[3], D, n_sys, pl.nseg, pl.sys, nsc, elem)))
        return 0;
    TileArgs a = {};
    a.X = X;
    a.n_sys = n_sys;
    a.n_row = n_row;
    a.nseg = pl.nseg;
    a.cl = pl.cl;
    a.nst = pl.nst;
    a.n_groups = (n_sys + pl.sys - 1) / pl.sys;
    a.accumulate = accumulate ? 1 : 0;
    a.gate = gate;
    a.status = status;
    const int rc = launch_tile_plan<TIN, TC>(pl, maps, a, cyclic, st);
    return rc == BTDMA_OK ? 1 : rc;
}

// Generated-coefficient batch, only D read (the GEN modes of the tiled
// kernel; the coefficient fields of `gen` are used, the rest is filled here).
// Returns 1 when launched, 0 when the shape is not tiled, < 0 on error.
// GEN 1 and 3 (one matrix for every system): `tab` is device scratch of
// n_row * 5 + (n_row / 16) * 6 doubles for the shared elimination factors.
template <int GEN, bool CYC = false>
int try_tile_gen(const double* D, double* X, int n_sys, int n_row, const TileArgs& gen,
                 unsigned* status, cudaStream_t st, double* tab = nullptr) {
    const TilePlan pl = tile_plan(n_row, CYC, 8, 1, GEN == 1 || GEN == 3);
    if (pl.sys == 0 || !tma_ok_elem(D, n_sys, 8)) return 0;
    const int nsc = pl.nseg / pl.cl;
    CUtensorMap maps[4];
    if (!make_tile_map(&maps[3], D, n_sys, pl.nseg, pl.sys, nsc, 8)) return 0;
    maps[0] = maps[1] = maps[2] = maps[3];  // not read in this mode
    TileArgs a = gen;
    a.X = X;
    a.n_sys = n_sys;
    a.n_row = n_row;
    a.nseg = pl.nseg;
    a.cl = pl.cl;
    a.nst = pl.nst;
    a.n_groups = (n_sys + pl.sys - 1) / pl.sys;
    a.accumulate = 0;
    a.gate = nullptr;
    a.status = status;
    if constexpr (GEN == 1 || GEN == 3) {
        if (!tab) return fail(BTDMA_ERR_ARG, "shared-matrix sweep without a factor table");
        tile_table_kernel<GEN><<<(pl.nseg + 127) / 128, 128, 0, st>>>(a, tab);
        CK(cudaGetLastError());
        a.gtab = tab;
    }
    int rc;
    switch (pl.sys) {
        case 128: rc = launch_tile_sys<128, CYC, double, double, GEN>(maps, a, st); break;
        case 64: rc = launch_tile_sys<64, CYC, double, double, GEN>(maps, a, st); break;
        case 32: rc = launch_tile_sys<32, CYC, double, double, GEN>(maps, a, st); break;
        default: rc = launch_tile_sys<16, CYC, double, double, GEN>(maps, a, st); break;
    }
    return rc == BTDMA_OK ? 1 : rc;
}

// Heat sweep: every row -cs, 1 + 2 cs, -cs; cs more on the diagonal of the
// first and last row when cbound.
int try_tile_const(const double* D, double* X, int n_sys, int n_row, double cs, bool cbound,
                   unsigned* status, cudaStream_t st, double* tab) {
    TileArgs g = {};
    g.cs = cs;
    g.cbound = cbound ? 1 : 0;
    return try_tile_gen<1>(D, X, n_sys, n_row, g, status, st, tab);
}

size_t gen_table_doubles(int n_row) { return (size_t)n_row * 5 + (size_t)(n_row / 16 + 1) * 6; }

template <bool CYCLIC>
int launch_seg_method(int method, const CUtensorMap* maps, const SegArgs& a, int groups,
                      cudaStream_t st) {
    switch (method) {
        case BTDMA_PASCAL: return launch_seg<SEG_PASCAL, CYCLIC>(maps, a, groups, st);
        case BTDMA_FILTERED_V1: return launch_seg<SEG_FILT_V1, CYCLIC>(maps, a, groups, st);
        default: return launch_seg<SEG_FILT_V2, CYCLIC>(maps, a, groups, st);
    }
}

int jmax_launch(btdma_t h, const double* D, int n_sys, int n_row, cudaStream_t st) {
    int blocks = std::max(1, std::min((n_sys + JRED_BLOCK - 1) / JRED_BLOCK, 1184 / h->P + 1));
    jmax_kernel<<<dim3(blocks, h->P), JRED_BLOCK, 0, st>>>(
        D, n_sys, n_row, h->P, (h->flags & BTDMA_FLAG_J_HOST) ? 1 : 0, h->work);
    CK(cudaGetLastError());
    return BTDMA_OK;
}

int jfinal_launch(btdma_t h, int n_row, int version, cudaStream_t st) {
    jfinal_kernel<<<1, 32, 0, st>>>(h->work, h->J, h->rho_row, n_row, h->P, h->eps_constant,
                                    version, (h->flags & BTDMA_FLAG_J_HOST) ? 1 : 0);
    CK(cudaGetLastError());
    return BTDMA_OK;
}

int check_sizes(btdma_t h, int n_sys, int n_row) {
    if (!h) return fail(BTDMA_ERR_ARG, "null handle");
    if (n_sys <= 0 || n_row <= 0) return fail(BTDMA_ERR_ARG, "n_sys and n_row must be positive");
    if (n_sys > h->n_sys_cap || n_row > h->n_row_cap)
        return fail(BTDMA_ERR_SIZE, "batch %d x %d exceeds the handle's %d x %d", n_row, n_sys,
                    h->n_row_cap, h->n_sys_cap);
    if (h->P > 1 && n_row / h->P < 3)
        return fail(BTDMA_ERR_SEGMENT, "n_row %d gives segments shorter than 3 rows at P=%d", n_row,
                    h->P);
    return BTDMA_OK;
}

int solve_impl(btdma_t h, const double* A, const double* B, const double* C, const double* D,
               double* X, int n_sys, int n_row, bool cyclic, cudaStream_t st) {
    int rc = check_sizes(h, n_sys, n_row);
    if (rc) return rc;
    if (!A || !B || !C || !D || !X) return fail(BTDMA_ERR_ARG, "null array");
    if (h->precision != BTDMA_FP64)
        return fail(BTDMA_ERR_UNSUPPORTED, "FP64 arrays passed to an FP32-refine handle");
    h->last_stream = st;

    if (h->P == 1) {
        if (cyclic && n_row < 3) return fail(BTDMA_ERR_ARG, "periodic systems need n_row >= 3");
        const int grid = (n_sys + THOMAS_BLOCK - 1) / THOMAS_BLOCK;
        double* Cs = h->scratch;
        double* Es = h->scratch + (size_t)h->n_row_cap * h->n_sys_cap;
        if (cyclic)
            thomas_cyclic_f64_kernel<<<grid, THOMAS_BLOCK, 0, st>>>(A, B, C, D, X, Cs, Es, n_sys,
                                                                    n_row, h->status);
        else
            thomas_f64_kernel<<<grid, THOMAS_BLOCK, 0, st>>>(A, B, C, D, X, Cs, n_sys, n_row,
                                                             h->status);
        CK(cudaGetLastError());
        return BTDMA_OK;
    }

    if (h->method == BTDMA_PASCAL && !(h->flags & BTDMA_FLAG_REFERENCE_ORDER)) {
        rc = try_tile<double>(A, B, C, D, X, n_sys, n_row, cyclic, h->status, st);
        if (rc < 0) return rc;
        if (rc == 1) return BTDMA_OK;
    }

    SegArgs a = {};
    a.A = A;
    a.B = B;
    a.C = C;
    a.D = D;
    a.X = X;
    a.n_sys = n_sys;
    a.n_row = n_row;
    a.P = h->P;
    a.mcap = seg_mcap(n_row, h->P);
    a.J = h->J;
    a.bnd = h->work;
    a.status = h->status;
    a.mode = SEG_MODE_SOLVE;
    if (seg_smem_bytes(a.mcap, a.P, cyclic) > (size_t)max_smem_optin())
        return fail(BTDMA_ERR_UNSUPPORTED,
                    "segment of %d rows does not fit in shared memory; use more segments",
                    a.mcap);
    CUtensorMap maps[5];
    std::memset(maps, 0, sizeof maps);
    a.use_tma = tma_ok(A, n_sys) && tma_ok(B, n_sys) && tma_ok(C, n_sys) && tma_ok(D, n_sys) &&
                tma_ok(X, n_sys);
    if (a.use_tma)
        a.use_tma = make_map(&maps[0], A, n_sys, n_row) && make_map(&maps[1], B, n_sys, n_row) &&
                    make_map(&maps[2], C, n_sys, n_row) && make_map(&maps[3], D, n_sys, n_row) &&
                    make_map(&maps[4], X, n_sys, n_row);
    const int groups = (n_sys + SEG_S - 1) / SEG_S;
    if (groups > 65535) return fail(BTDMA_ERR_SIZE, "n_sys above %d", 65535 * SEG_S);

    if (h->method == BTDMA_FILTERED_V2) {
        if ((rc = jmax_launch(h, D, n_sys, n_row, st))) return rc;
        if ((rc = jfinal_launch(h, n_row, 2, st))) return rc;
    } else if (h->method == BTDMA_FILTERED_V1) {
        SegArgs ai = a;
        ai.mode = SEG_MODE_INTERFACE;
        rc = cyclic ? launch_seg_method<true>(h->method, maps, ai, groups, st)
                    : launch_seg_method<false>(h->method, maps, ai, groups, st);
        if (rc) return rc;
        if ((rc = jfinal_launch(h, n_row, 1, st))) return rc;
    }
    return cyclic ? launch_seg_method<true>(h->method, maps, a, groups, st)
                  : launch_seg_method<false>(h->method, maps, a, groups, st);
}

}  // namespace

extern "C" {

const char* btdma_last_error(void) { return g_err.c_str(); }

int btdma_create(int method, int n_sys, int n_row, int P, int precision, int flags,
                 btdma_t* out) {
    if (!out) return fail(BTDMA_ERR_ARG, "null output handle");
    *out = nullptr;
    if (method < BTDMA_PASCAL || method > BTDMA_FILTERED_V2)
        return fail(BTDMA_ERR_ARG, "unknown method %d", method);
    if (n_sys <= 0 || n_row <= 0) return fail(BTDMA_ERR_ARG, "n_sys and n_row must be positive");
    if (precision < BTDMA_FP64 || precision > BTDMA_FP32_STORE)
        return fail(BTDMA_ERR_ARG, "unknown precision %d", precision);
    if (P < 0) return fail(BTDMA_ERR_ARG, "P must be >= 0");
    if (P == 0) P = auto_segments(n_row);
    if (P > SEG_MAX_P)
        return fail(BTDMA_ERR_UNSUPPORTED, "P=%d above the cluster limit %d", P, SEG_MAX_P);
    if (P > 1 && n_row / P < 3)
        return fail(BTDMA_ERR_SEGMENT, "n_row %d gives segments shorter than 3 rows at P=%d",
                    n_row, P);
    const bool tiled = method == BTDMA_PASCAL && !(flags & BTDMA_FLAG_REFERENCE_ORDER) &&
                       tile_plan(n_row, false).sys != 0;
    if (P > 1 && !tiled && seg_smem_bytes(seg_mcap(n_row, P), P, true) > (size_t)max_smem_optin())
        return fail(BTDMA_ERR_UNSUPPORTED, "segments of %d rows exceed shared memory; raise P",
                    (n_row + P - 1) / P);

    btdma_handle* h = new btdma_handle();
    h->method = method;
    h->P = P;
    h->precision = precision;
    h->flags = flags;
    h->n_sys_cap = n_sys;
    h->n_row_cap = n_row;
    h->eps_constant = 1.0e-12;
    auto cleanup = [&](int code) {
        btdma_destroy(h);
        return code;
    };
#define CKC(call)                                                                                \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return cleanup(fail(BTDMA_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)));       \
    } while (0)
    CKC(cudaMalloc(&h->rho_row, sizeof(double) * n_row));
    CKC(cudaMemset(h->rho_row, 0, sizeof(double) * n_row));
    CKC(cudaMalloc(&h->J, sizeof(int) * P));
    CKC(cudaMemset(h->J, 0, sizeof(int) * P));
    CKC(cudaMalloc(&h->work, sizeof(unsigned long long) * 2 * P));
    CKC(cudaMemset(h->work, 0, sizeof(unsigned long long) * 2 * P));
    CKC(cudaMalloc(&h->status, sizeof(unsigned)));
    CKC(cudaMemset(h->status, 0, sizeof(unsigned)));
    if (P == 1 && precision == BTDMA_FP64)
        CKC(cudaMalloc(&h->scratch, sizeof(double) * 2 * (size_t)n_row * n_sys));
    if (precision == BTDMA_FP32_REFINE) {
        CKC(cudaMalloc(&h->resid, sizeof(float) * (size_t)n_row * n_sys));
        CKC(cudaMalloc(&h->iters, (size_t)n_sys));
        CKC(cudaMalloc(&h->open, sizeof(unsigned) * (BTDMA_REFINE_MAX_SWEEPS + 1)));
    }
#undef CKC
    *out = h;
    return BTDMA_OK;
}

int btdma_destroy(btdma_t h) {
    if (!h) return BTDMA_OK;
    cudaFree(h->rho_row);
    cudaFree(h->J);
    cudaFree(h->work);
    cudaFree(h->status);
    cudaFree(h->scratch);
    cudaFree(h->resid);
    cudaFree(h->iters);
    cudaFree(h->open);
    cudaFree(h->rag_d_off);
    cudaFree(h->rag_d_list);
    cudaFree(h->rag_d_tasks);
    cudaFree(h->rag_d_probe);
    for (int i = 0; i < btdma_handle::RAG_STREAMS; ++i) {
        if (h->rag_side[i]) cudaStreamDestroy(h->rag_side[i]);
        if (h->rag_join[i]) cudaEventDestroy(h->rag_join[i]);
    }
    if (h->rag_fork) cudaEventDestroy(h->rag_fork);
    delete h;
    return BTDMA_OK;
}

int btdma_solve(btdma_t h, const double* A, const double* B, const double* C, double* D,
                int n_sys, int n_row, cudaStream_t stream) {
    return solve_impl(h, A, B, C, D, D, n_sys, n_row, false, stream);
}

int btdma_solve_cyclic(btdma_t h, const double* A, const double* B, const double* C, double* D,
                       int n_sys, int n_row, cudaStream_t stream) {
    return solve_impl(h, A, B, C, D, D, n_sys, n_row, true, stream);
}

int btdma_solve_out(btdma_t h, const double* A, const double* B, const double* C,
                    const double* D, double* X, int n_sys, int n_row, int cyclic,
                    cudaStream_t stream) {
    return solve_impl(h, A, B, C, D, X, n_sys, n_row, cyclic != 0, stream);
}

int btdma_solve_f32(btdma_t h, const float* A, const float* B, const float* C, const float* D,
                    double* X, int n_sys, int n_row, int cyclic, cudaStream_t stream) {
    int rc = check_sizes(h, n_sys, n_row);
    if (rc) return rc;
    if (!A || !B || !C || !D || !X) return fail(BTDMA_ERR_ARG, "null array");
    if (h->precision != BTDMA_FP32_STORE && h->precision != BTDMA_FP32_REFINE)
        return fail(BTDMA_ERR_ARG, "FP32 arrays passed to an FP64 handle");
    if (h->method != BTDMA_PASCAL)
        return fail(BTDMA_ERR_UNSUPPORTED, "FP32 storage is provided for PaScaL only");
    h->last_stream = stream;
    h->last_n_sys = n_sys;
    h->last_refined = false;
    const bool cyc = cyclic != 0;
    const char* shape_msg =
        "FP32 storage needs n_row % 16 == 0, n_sys % 4 == 0, 16-byte alignment "
        "(and a power-of-two n_row/16 when periodic)";
    if (h->precision == BTDMA_FP32_STORE) {
        rc = try_tile<float>(A, B, C, D, X, n_sys, n_row, cyc, h->status, stream);
        if (rc < 0) return rc;
        if (rc == 0) return fail(BTDMA_ERR_UNSUPPORTED, "%s", shape_msg);
        return BTDMA_OK;
    }
    // FP32_REFINE: x0 from the FP32 sweeps, then up to max_sweeps of
    //   r = D - T x (FP64), e = T^-1 r (FP32 sweeps), x += e,
    // each launch gated on the device count of still-open systems, so the whole
    // sequence is stream-ordered and capturable (no host round trip).
    const int S = h->max_sweeps;
    CK(cudaMemsetAsync(h->open, 0, sizeof(unsigned) * (BTDMA_REFINE_MAX_SWEEPS + 1), stream));
    rc = try_tile<float, float>(A, B, C, D, X, n_sys, n_row, cyc, h->status, stream);
    if (rc < 0) return rc;
    if (rc == 0) return fail(BTDMA_ERR_UNSUPPORTED, "%s", shape_msg);
    const int rgrid = (n_sys + 255) / 256;
    for (int s = 0; s <= S; ++s) {
        refine_residual_kernel<<<rgrid, 256, 0, stream>>>(
            A, B, C, D, X, h->resid, n_sys, n_row, cyclic ? 1 : 0, s, s == S ? 1 : 0, h->eta_tol,
            h->iters, s == 0 ? nullptr : &h->open[s - 1], &h->open[s]);
        CK(cudaGetLastError());
        if (s == S) break;
        rc = try_tile<float, float>(A, B, C, h->resid, X, n_sys, n_row, cyc, h->status, stream,
                                    true, &h->open[s]);
        if (rc < 0) return rc;
    }
    // fallback: the FP64-arithmetic solve of the whole batch while any system is open
    rc = try_tile<float, double>(A, B, C, D, X, n_sys, n_row, cyc, h->status, stream, false,
                                 &h->open[S]);
    if (rc < 0) return rc;
    h->last_refined = true;
    return BTDMA_OK;
}

int btdma_set_refine(btdma_t h, int max_sweeps, double eta_tol) {
    if (!h) return fail(BTDMA_ERR_ARG, "null handle");
    if (max_sweeps < 0 || max_sweeps > BTDMA_REFINE_MAX_SWEEPS)
        return fail(BTDMA_ERR_ARG, "max_sweeps must be in [0, %d]", BTDMA_REFINE_MAX_SWEEPS);
    if (!(eta_tol > 0.0)) return fail(BTDMA_ERR_ARG, "eta_tol must be positive");
    h->max_sweeps = max_sweeps;
    h->eta_tol = eta_tol;
    return BTDMA_OK;
}

int btdma_last_stats(btdma_t h, btdma_stats* st) {
    if (!h || !st) return fail(BTDMA_ERR_ARG, "null argument");
    std::memset(st, 0, sizeof *st);
    st->n_systems = h->last_n_sys;
    if (!h->last_refined) return BTDMA_OK;
    std::vector<unsigned char> it((size_t)h->last_n_sys);
    unsigned open[BTDMA_REFINE_MAX_SWEEPS + 1];
    CK(cudaMemcpyAsync(it.data(), h->iters, it.size(), cudaMemcpyDeviceToHost, h->last_stream));
    CK(cudaMemcpyAsync(open, h->open, sizeof open, cudaMemcpyDeviceToHost, h->last_stream));
    CK(cudaStreamSynchronize(h->last_stream));
    for (unsigned char v : it) {
        if (v == REFINE_FALLBACK || v == REFINE_OPEN)
            ++st->n_fallback;
        else if (v <= BTDMA_REFINE_MAX_SWEEPS)
            ++st->converged_after[v];
    }
    // a correction sweep ran when systems were open before it
    for (int s = 0; s < h->max_sweeps; ++s)
        if (open[s] != 0u) st->sweeps = s + 1;
    return BTDMA_OK;
}

int btdma_set_eps_constant(btdma_t h, double eps_constant) {
    if (!h) return fail(BTDMA_ERR_ARG, "null handle");
    h->eps_constant = eps_constant;
    return BTDMA_OK;
}

int btdma_set_rho(btdma_t h, const double* A, const double* B, const double* C, int n_sys,
                  int n_row, cudaStream_t stream) {
    int rc = check_sizes(h, n_sys, n_row);
    if (rc) return rc;
    if (h->method == BTDMA_PASCAL) return BTDMA_OK;
    rho_sys0_kernel<<<(n_row + 255) / 256, 256, 0, stream>>>(A, B, C, n_sys, n_row, h->rho_row);
    CK(cudaGetLastError());
    return BTDMA_OK;
}

int btdma_set_rho_all(btdma_t h, const double* A, const double* B, const double* C, int n_sys,
                      int n_row, cudaStream_t stream) {
    int rc = check_sizes(h, n_sys, n_row);
    if (rc) return rc;
    if (h->method == BTDMA_PASCAL) return BTDMA_OK;
    CK(cudaMemsetAsync(h->rho_row, 0, sizeof(double) * n_row, stream));
    int bx = std::max(1, std::min((n_sys + 255) / 256, 32));
    rho_all_kernel<<<dim3(bx, n_row), 256, 0, stream>>>(
        A, B, C, n_sys, reinterpret_cast<unsigned long long*>(h->rho_row));
    CK(cudaGetLastError());
    return BTDMA_OK;
}

int btdma_last_J(btdma_t h, int* J, int cap, int* n_out) {
    if (!h) return fail(BTDMA_ERR_ARG, "null handle");
    if (n_out) *n_out = h->P;
    if (!J || cap <= 0) return BTDMA_OK;
    const int n = std::min(cap, h->P);
    if (h->P == 1 || h->method == BTDMA_PASCAL) {
        for (int k = 0; k < n; ++k) J[k] = -1;
        return BTDMA_OK;
    }
    CK(cudaMemcpyAsync(J, h->J, sizeof(int) * n, cudaMemcpyDeviceToHost, h->last_stream));
    CK(cudaStreamSynchronize(h->last_stream));
    return BTDMA_OK;
}

int btdma_status(btdma_t h, unsigned* status) {
    if (!h || !status) return fail(BTDMA_ERR_ARG, "null argument");
    CK(cudaMemcpyAsync(status, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost,
                       h->last_stream));
    CK(cudaStreamSynchronize(h->last_stream));
    CK(cudaMemsetAsync(h->status, 0, sizeof(unsigned), h->last_stream));
    CK(cudaStreamSynchronize(h->last_stream));
    return BTDMA_OK;
}

int btdma_set_method(btdma_t h, int method) {
    if (!h) return fail(BTDMA_ERR_ARG, "null handle");
    if (method < BTDMA_PASCAL || method > BTDMA_FILTERED_V2)
        return fail(BTDMA_ERR_ARG, "unknown method %d", method);
    h->method = method;
    return BTDMA_OK;
}

int btdma_segments(btdma_t h, int* P) {
    if (!h || !P) return fail(BTDMA_ERR_ARG, "null argument");
    *P = h->P;
    return BTDMA_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free serial Thomas (btdma_solve_noalloc).  The forward sweep's c'
// goes to this fixed device array instead of handle-owned scratch.  Host code
// may not pass the array's name to a kernel (on the host it is only a
// stand-in symbol), so its device address is looked up once per device with
// that device current and cached here.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_noalloc_scratch[BTDMA_NOALLOC_MAX_ELEMS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kMaxDevices] = {};

int noalloc_scratch(double** out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(BTDMA_ERR_UNSUPPORTED, "device %d", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return BTDMA_OK;
}

}  // namespace

extern "C" int btdma_solve_noalloc(const double* A, const double* B, const double* C, double* D,
                                   int n_sys, int n_row, cudaStream_t stream) {
    if (!A || !B || !C || !D) return fail(BTDMA_ERR_ARG, "null array");
    if (n_sys <= 0 || n_row <= 0) return fail(BTDMA_ERR_ARG, "n_sys and n_row must be positive");
    if ((long long)n_sys * n_row > (long long)BTDMA_NOALLOC_MAX_ELEMS)
        return fail(BTDMA_ERR_SIZE,
                    "n_sys * n_row = %lld exceeds the allocation-free limit of %d elements",
                    (long long)n_sys * n_row, BTDMA_NOALLOC_MAX_ELEMS);
    double* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    // c' is written before it is read by the same thread, so the scratch needs
    // no clearing between calls.
    const int grid = (n_sys + THOMAS_BLOCK - 1) / THOMAS_BLOCK;
    thomas_f64_kernel<<<grid, THOMAS_BLOCK, 0, stream>>>(A, B, C, D, D, scratch, n_sys, n_row,
                                                         nullptr);
    CK(cudaGetLastError());
    return BTDMA_OK;
}


// ------------------------------------------------------------------ ragged
namespace {

constexpr int RAG_WPC = 4;         // warps per CTA of the warp-kind launch
constexpr int RAG_WARP_MCAP = 32;  // rows per lane the warp kind accepts

// Lanes per system for a bucket whose systems have nmin..nmax rows: about
// 12 rows per lane, a power of two, at most 32, and at least 3 rows per lane
// for the shortest system.
int rag_default_P(int nmin, int nmax) {
    int P = 1;
    while (P < 32 && nmax / (2 * P) >= 12 && nmin / (2 * P) >= 3) P <<= 1;
    return P;
}

int rag_mcap(int nmax, int P) { return (nmax + P - 1) / P; }

// CTA-per-system shape for long systems: the smallest power of two >= 64 that
// keeps <= RAG_MT rows per thread (0 when none <= 512 does, or when the
// shortest system would get fewer than 3 rows per thread).
int rag_cta_P(int nmin, int nmax) {
    int P = 64;
    while (P <= 512 && rag_mcap(nmax, P) > RAG_MT) P <<= 1;
    return (P <= 512 && nmin / P >= 3) ? P : 0;
}

// Task entries of one bucket with lanes-per-system P (warp kind: 32 / P
// systems per warp; CTA kind: one system per CTA).
void rag_bucket_tasks(const btdma_handle::RagBucket& b, int cta, int P, std::vector<int4>& out) {
    if (cta) {
        for (int i = 0; i < b.count; ++i) out.push_back(make_int4(b.first + i, b.cyc, 0, 0));
        return;
    }
    const int G = 32 / P;
    for (int i = 0; i < b.count; i += G)
        out.push_back(make_int4(b.first + i, std::min(G, b.count - i), P, b.cyc));
}

// Task tables of the whole plan: one warp-kind launch (buckets longest first)
// and one CTA-kind launch per P.
int rag_build_launches(btdma_t h) {
    std::vector<int4> tasks;
    h->rag_launches.clear();
    btdma_handle::RagLaunch wl{0, 0, 0, 0, 1, 0};
    for (int i = (int)h->rag_buckets.size() - 1; i >= 0; --i) {
        const auto& b = h->rag_buckets[i];
        if (b.cta) continue;
        rag_bucket_tasks(b, 0, b.P, tasks);
        wl.mcap = std::max(wl.mcap, rag_mcap(b.nmax, b.P));
    }
    wl.count = (int)tasks.size();
    if (wl.count) h->rag_launches.push_back(wl);
    for (int P = 512; P >= 64; P >>= 1)
        for (int stg = 0; stg < 2; ++stg) {
            btdma_handle::RagLaunch cl{1, P, (int)tasks.size(), 0, 0, stg};
            for (const auto& b : h->rag_buckets)
                if (b.cta && b.P == P && b.staged == stg) rag_bucket_tasks(b, 1, P, tasks);
            cl.count = (int)tasks.size() - cl.first;
            if (cl.count) h->rag_launches.push_back(cl);
        }
    CK(cudaMemcpy(h->rag_d_tasks, tasks.data(), sizeof(int4) * tasks.size(),
                  cudaMemcpyHostToDevice));
    return BTDMA_OK;
}

int rag_plan(btdma_t h, const long long* off, const unsigned char* per, int n_sys) {
    if (n_sys <= 0) return fail(BTDMA_ERR_ARG, "n_sys must be positive");
    if (!off) return fail(BTDMA_ERR_ARG, "null row offsets");
    if (off[0] != 0) return fail(BTDMA_ERR_ARG, "row_offsets[0] must be 0");
    const bool same = (int)h->rag_off.size() == n_sys + 1 &&
                      std::equal(off, off + n_sys + 1, h->rag_off.begin()) &&
                      (per ? (h->rag_per.size() == (size_t)n_sys &&
                              std::equal(per, per + n_sys, h->rag_per.begin()))
                           : h->rag_per.empty());
    if (same && h->rag_d_off) return BTDMA_OK;
    // bucket key: (periodic, ceil(log2 n))
    std::vector<int> key(n_sys);
    for (int i = 0; i < n_sys; ++i) {
        const long long n = off[i + 1] - off[i];
        if (n < 3) return fail(BTDMA_ERR_SEGMENT, "system %d has %lld rows (needs >= 3)", i, n);
        if (n > 32 * RAG_WARP_MCAP && n > 512 * RAG_MT)
            return fail(BTDMA_ERR_SIZE, "system %d has %lld rows (at most %d)", i, n,
                        512 * RAG_MT);
        int lg = 0;
        while ((1LL << lg) < n) ++lg;
        key[i] = (per && per[i] ? 64 : 0) + lg;
    }
    std::vector<int> order(n_sys);
    for (int i = 0; i < n_sys; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return key[x] < key[y]; });
    std::vector<btdma_handle::RagBucket> bk;
    for (int i = 0; i < n_sys;) {
        int j = i;
        int nmin = INT32_MAX, nmax = 0;
        while (j < n_sys && key[order[j]] == key[order[i]]) {
            const int n = (int)(off[order[j] + 1] - off[order[j]]);
            nmin = std::min(nmin, n);
            nmax = std::max(nmax, n);
            ++j;
        }
        btdma_handle::RagBucket b{};
        b.cyc = key[order[i]] >= 64 ? 1 : 0;
        b.first = i;
        b.count = j - i;
        b.nmin = nmin;
        b.nmax = nmax;
        const int Pc = nmax > 32 * RAG_MT ? rag_cta_P(nmin, nmax) : 0;
        if (Pc) {
            b.cta = 1;
            b.P = Pc;
        } else {
            b.cta = 0;
            b.P = rag_default_P(nmin, nmax);
            if (rag_mcap(nmax, b.P) > RAG_WARP_MCAP)
                return fail(BTDMA_ERR_UNSUPPORTED, "no launch shape for systems of %d..%d rows",
                            nmin, nmax);
        }
        b.warps = b.cta ? b.P / 32 : RAG_WPC;
        b.mcap = rag_mcap(nmax, b.P);
        b.best_ms = 0.f;
        bk.push_back(b);
        i = j;
    }
    cudaFree(h->rag_d_off);
    cudaFree(h->rag_d_list);
    cudaFree(h->rag_d_tasks);
    cudaFree(h->rag_d_probe);
    h->rag_d_off = nullptr;
    h->rag_d_list = nullptr;
    h->rag_d_tasks = h->rag_d_probe = nullptr;
    h->rag_off.clear();
    CK(cudaMalloc(&h->rag_d_off, sizeof(long long) * (n_sys + 1)));
    CK(cudaMalloc(&h->rag_d_list, sizeof(int) * n_sys));
    CK(cudaMalloc(&h->rag_d_tasks, sizeof(int4) * 2 * n_sys));
    CK(cudaMalloc(&h->rag_d_probe, sizeof(int4) * n_sys));
    CK(cudaMemcpy(h->rag_d_off, off, sizeof(long long) * (n_sys + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->rag_d_list, order.data(), sizeof(int) * n_sys, cudaMemcpyHostToDevice));
    if (!h->rag_fork) {
        CK(cudaEventCreateWithFlags(&h->rag_fork, cudaEventDisableTiming));
        for (int i = 0; i < btdma_handle::RAG_STREAMS; ++i) {
            CK(cudaStreamCreateWithFlags(&h->rag_side[i], cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&h->rag_join[i], cudaEventDisableTiming));
        }
    }
    h->rag_buckets = bk;
    h->rag_order = order;
    const int rc = rag_build_launches(h);
    if (rc) return rc;
    h->rag_off.assign(off, off + n_sys + 1);
    if (per)
        h->rag_per.assign(per, per + n_sys);
    else
        h->rag_per.clear();
    return BTDMA_OK;
}

template <typename TIN>
int rag_launch(btdma_t h, int cta, int P, int mcap, int staged, const int4* tasks, int n_tasks,
               const TIN* A, const TIN* B, const TIN* C, const TIN* D, double* X,
               cudaStream_t st) {
    RagArgs a{};
    a.A = A;
    a.B = B;
    a.C = C;
    a.D = D;
    a.X = X;
    a.off = h->rag_d_off;
    a.list = h->rag_d_list;
    a.tasks = tasks;
    a.n_tasks = n_tasks;
    a.mcap = mcap;
    a.status = h->status;
    if (cta) {
        if (staged && rag_cta_smem_bytes(P, true) > (size_t)max_smem_optin()) staged = 0;
        auto kern = staged ? ragged_cta_kernel<TIN, true> : ragged_cta_kernel<TIN, false>;
        static bool attr_done[2] = {false, false};
        if (!attr_done[staged]) {
            CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    max_smem_optin()));
            attr_done[staged] = true;
        }
        kern<<<n_tasks, P, rag_cta_smem_bytes(P, staged), st>>>(a);
    } else {
        auto kern = ragged_kernel<TIN>;
        static bool attr_done = false;
        if (!attr_done) {
            CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    max_smem_optin()));
            attr_done = true;
        }
        kern<<<(n_tasks + RAG_WPC - 1) / RAG_WPC, 32 * RAG_WPC, rag_smem_bytes(RAG_WPC, mcap),
               st>>>(a);
    }
    CK(cudaGetLastError());
    return BTDMA_OK;
}

// All launches of the plan: the first on the caller's stream, the others on
// side streams forked from it and joined back (graph-capturable).
template <typename TIN>
int rag_run(btdma_t h, const TIN* A, const TIN* B, const TIN* C, const TIN* D, double* X,
            cudaStream_t st) {
    const auto& L = h->rag_launches;
    const int n = (int)L.size();
    const int side = std::min(n - 1, (int)btdma_handle::RAG_STREAMS);
    if (side > 0) {
        CK(cudaEventRecord(h->rag_fork, st));
        for (int i = 0; i < side; ++i) CK(cudaStreamWaitEvent(h->rag_side[i], h->rag_fork, 0));
    }
    for (int i = 0; i < n; ++i) {
        const cudaStream_t s = i == 0 ? st : h->rag_side[(i - 1) % btdma_handle::RAG_STREAMS];
        const int rc = rag_launch<TIN>(h, L[i].cta, L[i].P, L[i].mcap, L[i].staged,
                                       h->rag_d_tasks + L[i].first, L[i].count, A, B, C, D, X,
                                       s);
        if (rc) return rc;
    }
    for (int i = 0; i < side; ++i) {
        CK(cudaEventRecord(h->rag_join[i], h->rag_side[i]));
        CK(cudaStreamWaitEvent(st, h->rag_join[i], 0));
    }
    return BTDMA_OK;
}

template <typename TIN>
int rag_solve(btdma_t h, const TIN* A, const TIN* B, const TIN* C, const TIN* D, double* X,
              const long long* off, const unsigned char* per, int n_sys, cudaStream_t st) {
    if (!h) return fail(BTDMA_ERR_ARG, "null handle");
    if (!A || !B || !C || !D || !X) return fail(BTDMA_ERR_ARG, "null array");
    if (h->method != BTDMA_PASCAL)
        return fail(BTDMA_ERR_UNSUPPORTED, "ragged batches are solved by PaScaL only");
    const bool f32 = sizeof(TIN) == 4;
    if (f32 != (h->precision != BTDMA_FP64))
        return fail(BTDMA_ERR_ARG, "array type does not match the handle's precision");
    int rc = rag_plan(h, off, per, n_sys);
    if (rc) return rc;
    h->last_stream = st;
    h->last_n_sys = n_sys;
    h->last_refined = false;
    return rag_run<TIN>(h, A, B, C, D, X, st);
}

// Times, bucket by bucket, every launch shape on the given batch (the bucket
// alone, best of 3, CUDA events on the stream) and keeps the fastest; then
// rebuilds the merged task tables.  X is overwritten.
template <typename TIN>
int rag_tune(btdma_t h, const TIN* A, const TIN* B, const TIN* C, const TIN* D, double* X,
             const long long* off, const unsigned char* per, int n_sys, cudaStream_t st) {
    int rc = rag_solve<TIN>(h, A, B, C, D, X, off, per, n_sys, st);  // plan + warm-up
    if (rc) return rc;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    std::vector<int4> tasks;
    for (auto& b : h->rag_buckets) {
        struct Cand {
            int cta, P, staged;
        };
        std::vector<Cand> cands;
        for (int P = 1; P <= 32 && b.nmin / P >= 3; P <<= 1)
            if (rag_mcap(b.nmax, P) <= RAG_WARP_MCAP) cands.push_back({0, P, 0});
        for (int P = 64; P <= 512 && b.nmin / P >= 3; P <<= 1)
            if (rag_mcap(b.nmax, P) <= RAG_MT) {
                cands.push_back({1, P, 0});
                if (rag_cta_smem_bytes(P, true) <= (size_t)max_smem_optin())
                    cands.push_back({1, P, 1});
            }
        float best = 1e30f;
        Cand pick{b.cta, b.P, b.staged};
        for (const Cand& cd : cands) {
            tasks.clear();
            rag_bucket_tasks(b, cd.cta, cd.P, tasks);
            if (cudaMemcpyAsync(h->rag_d_probe, tasks.data(), sizeof(int4) * tasks.size(),
                                cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                rc = fail(BTDMA_ERR_CUDA, "autotune upload failed");
                break;
            }
            float ms = 0.f;
            for (int rep = 0; rep < 3 && !rc; ++rep) {
                CK(cudaEventRecord(e0, st));
                rc = rag_launch<TIN>(h, cd.cta, cd.P, rag_mcap(b.nmax, cd.P), cd.staged,
                                     h->rag_d_probe, (int)tasks.size(), A, B, C, D, X, st);
                if (rc) break;
                CK(cudaEventRecord(e1, st));
                CK(cudaEventSynchronize(e1));
                float t = 0.f;
                CK(cudaEventElapsedTime(&t, e0, e1));
                ms = rep == 0 ? t : std::min(ms, t);
            }
            if (rc) break;
            if (ms < best) {
                best = ms;
                pick = cd;
            }
        }
        if (rc) break;
        b.cta = pick.cta;
        b.staged = pick.staged;
        b.P = pick.P;
        b.warps = pick.cta ? pick.P / 32 : RAG_WPC;
        b.mcap = rag_mcap(b.nmax, pick.P);
        b.best_ms = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    return rag_build_launches(h);
}

}  // namespace

int btdma_solve_ragged(btdma_t h, const double* A, const double* B, const double* C,
                       const double* D, double* X, const long long* row_offsets,
                       const unsigned char* is_periodic, int n_sys, cudaStream_t stream) {
    return rag_solve<double>(h, A, B, C, D, X, row_offsets, is_periodic, n_sys, stream);
}

int btdma_solve_ragged_f32(btdma_t h, const float* A, const float* B, const float* C,
                           const float* D, double* X, const long long* row_offsets,
                           const unsigned char* is_periodic, int n_sys, cudaStream_t stream) {
    return rag_solve<float>(h, A, B, C, D, X, row_offsets, is_periodic, n_sys, stream);
}

int btdma_ragged_autotune(btdma_t h, const void* A, const void* B, const void* C, const void* D,
                          double* X, const long long* row_offsets,
                          const unsigned char* is_periodic, int n_sys, cudaStream_t stream) {
    if (!h) return fail(BTDMA_ERR_ARG, "null handle");
    if (h->precision == BTDMA_FP64)
        return rag_tune<double>(h, static_cast<const double*>(A), static_cast<const double*>(B),
                                static_cast<const double*>(C), static_cast<const double*>(D), X,
                                row_offsets, is_periodic, n_sys, stream);
    return rag_tune<float>(h, static_cast<const float*>(A), static_cast<const float*>(B),
                           static_cast<const float*>(C), static_cast<const float*>(D), X,
                           row_offsets, is_periodic, n_sys, stream);
}

int btdma_ragged_plan_info(btdma_t h, btdma_ragged_bucket* out, int cap, int* n_out) {
    if (!h || !n_out) return fail(BTDMA_ERR_ARG, "null argument");
    *n_out = (int)h->rag_buckets.size();
    for (int i = 0; i < cap && i < *n_out; ++i) {
        const auto& b = h->rag_buckets[i];
        out[i].periodic = b.cyc;
        out[i].n_systems = b.count;
        out[i].n_row_min = b.nmin;
        out[i].n_row_max = b.nmax;
        out[i].lanes_per_system = b.P;
        out[i].warps_per_cta = b.warps;
        out[i].cta_per_system = b.cta + b.staged;
        out[i].tuned_ms = b.best_ms;
    }
    return BTDMA_OK;
}

// ------------------------------------------------------------- heat ADI step
struct btdma_heat {
    HeatGeom g{};
    double* xc = nullptr;  // device coordinates (ghosts included)
    double* yc = nullptr;
    double* zc = nullptr;
    double* cosx = nullptr;  // cos(pi x) etc. at the cell centres
    double* cosy = nullptr;
    double* cosz = nullptr;
    double* buf0 = nullptr;  // Z and X sweep layouts
    double* buf1 = nullptr;  // Y sweep layout
    double* err = nullptr;   // L2 accumulator
    double* scratch = nullptr;  // full grid, the warm-up step before graph capture
    double* tab = nullptr;      // shared elimination factors of one sweep
    unsigned* status = nullptr;
    cudaStream_t cap = nullptr;  // private stream the step graph is captured on
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double* graph_theta = nullptr;  // theta the graph was captured for
    cudaStream_t last_stream = nullptr;
};

namespace {

// One step as a kernel sequence on stream st (seven launches, no host sync).
int heat_enqueue(btdma_heat_t h, double* theta, cudaStream_t st) {
    const HeatGeom& g = h->g;
    const dim3 b1(128, 1, 1);
    const dim3 gr((g.ix + 127) / 128, g.iy, g.iz);
    heat_rhs_z_kernel<<<gr, b1, 0, st>>>(theta, h->buf0, g);
    CK(cudaGetLastError());
    int rc = try_tile_const(h->buf0, h->buf0, g.ix * g.iy, g.iz, g.bz, true, h->status, st, h->tab);
    if (rc != 1) return rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "Z sweep not tileable");
    heat_z_to_y_kernel<<<gr, b1, 0, st>>>(theta, h->buf0, h->buf1, g);
    CK(cudaGetLastError());
    rc = try_tile_const(h->buf1, h->buf1, g.ix * g.iz, g.iy, g.by, true, h->status, st, h->tab);
    if (rc != 1) return rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "Y sweep not tileable");
    const dim3 bt(HEAT_TILE, 8, 1);
    heat_y_to_x_kernel<<<dim3((g.ix + HEAT_TILE - 1) / HEAT_TILE, (g.iy + HEAT_TILE - 1) / HEAT_TILE,
                              g.iz), bt, 0, st>>>(theta, h->buf1, h->buf0, g);
    CK(cudaGetLastError());
    rc = try_tile_const(h->buf0, h->buf0, g.iy * g.iz, g.ix, g.bx, true, h->status, st, h->tab);
    if (rc != 1) return rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "X sweep not tileable");
    heat_update_kernel<<<dim3((g.iy + HEAT_TILE - 1) / HEAT_TILE, (g.ix + HEAT_TILE - 1) / HEAT_TILE,
                              g.iz), bt, 0, st>>>(theta, h->buf0, g);
    CK(cudaGetLastError());
    return BTDMA_OK;
}

}  // namespace

int btdma_heat_create(int ix, int iy, int iz, double dt, btdma_heat_t* out) {
    if (!out) return fail(BTDMA_ERR_ARG, "null output handle");
    *out = nullptr;
    if (ix <= 0 || iy <= 0 || iz <= 0 || !(dt > 0.0))
        return fail(BTDMA_ERR_ARG, "grid sizes and dt must be positive");
    if (ix % 16 || iy % 16 || iz % 16)
        return fail(BTDMA_ERR_UNSUPPORTED, "the fused step needs ix, iy, iz multiples of 16");
    if ((long long)(ix + 2) * (iy + 2) >= (1LL << 31) || (long long)ix * iy >= (1LL << 31) ||
        (long long)ix * iz >= (1LL << 31) || (long long)iy * iz >= (1LL << 31))
        return fail(BTDMA_ERR_SIZE, "grid planes above 2^31 cells");
    if (!tile_plan(iz, false, 8, 1).sys || !tile_plan(iy, false, 8, 1).sys ||
        !tile_plan(ix, false, 8, 1).sys)
        return fail(BTDMA_ERR_UNSUPPORTED, "grid not supported by the tiled solve");
    btdma_heat* h = new btdma_heat();
    auto cleanup = [&](int code) {
        btdma_heat_destroy(h);
        return code;
    };
#define CKH(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return cleanup(fail(BTDMA_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_))); \
    } while (0)
    // cell centres with one ghost each side, x_c[i] = x0 + dd/2 + (i - 1) dd on
    // [-1, 1] with dd = 2 / n (mpi_subdomain.cpp mesh(), one rank)
    auto coords = [](int n) {
        std::vector<double> c(n + 2);
        const double dd = 2.0 / n;
        for (int i = 0; i < n + 2; ++i) c[i] = -1.0 + dd / 2.0 + (i - 1) * dd;
        return c;
    };
    const auto hx = coords(ix), hy = coords(iy), hz = coords(iz);
    auto cosines = [](const std::vector<double>& c) {
        std::vector<double> o(c.size());
        for (size_t i = 0; i < c.size(); ++i) o[i] = std::cos(HEAT_PI * c[i]);
        return o;
    };
    const auto kx = cosines(hx), ky = cosines(hy), kz = cosines(hz);
    auto upload = [&](double** dst, const std::vector<double>& v) {
        cudaError_t e = cudaMalloc(dst, sizeof(double) * v.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(*dst, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice);
        return e;
    };
    CKH(upload(&h->xc, hx));
    CKH(upload(&h->yc, hy));
    CKH(upload(&h->zc, hz));
    CKH(upload(&h->cosx, kx));
    CKH(upload(&h->cosy, ky));
    CKH(upload(&h->cosz, kz));
    const size_t inner = (size_t)ix * iy * iz;
    CKH(cudaMalloc(&h->buf0, sizeof(double) * inner));
    CKH(cudaMalloc(&h->buf1, sizeof(double) * inner));
    CKH(cudaMalloc(&h->err, sizeof(double)));
    CKH(cudaMalloc(&h->scratch, sizeof(double) * (size_t)(ix + 2) * (iy + 2) * (iz + 2)));
    CKH(cudaMalloc(&h->tab, sizeof(double) * gen_table_doubles(std::max(ix, std::max(iy, iz)))));
    CKH(cudaMalloc(&h->status, sizeof(unsigned)));
    CKH(cudaMemset(h->status, 0, sizeof(unsigned)));
    CKH(cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking));
#undef CKH
    HeatGeom& g = h->g;
    g.ix = ix;
    g.iy = iy;
    g.iz = iz;
    g.dt = dt;
    const double dx = 2.0 / ix, dy = 2.0 / iy, dz = 2.0 / iz;
    g.bx = dt / (2.0 * dx * dx);  // stencil base, stencil_coeffs.hpp:10-13
    g.by = dt / (2.0 * dy * dy);
    g.bz = dt / (2.0 * dz * dz);
    g.xc = h->xc;
    g.yc = h->yc;
    g.zc = h->zc;
    g.cx = h->cosx;
    g.cy = h->cosy;
    g.cz = h->cosz;
    *out = h;
    return BTDMA_OK;
}

int btdma_heat_destroy(btdma_heat_t h) {
    if (!h) return BTDMA_OK;
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->cap) cudaStreamDestroy(h->cap);
    cudaFree(h->xc);
    cudaFree(h->yc);
    cudaFree(h->zc);
    cudaFree(h->cosx);
    cudaFree(h->cosy);
    cudaFree(h->cosz);
    cudaFree(h->buf0);
    cudaFree(h->buf1);
    cudaFree(h->err);
    cudaFree(h->scratch);
    cudaFree(h->tab);
    cudaFree(h->status);
    delete h;
    return BTDMA_OK;
}

int btdma_heat_init(btdma_heat_t h, double* theta, cudaStream_t stream) {
    if (!h || !theta) return fail(BTDMA_ERR_ARG, "null argument");
    const HeatGeom& g = h->g;
    heat_init_kernel<<<dim3((g.ix + 2 + 127) / 128, g.iy + 2, g.iz + 2), 128, 0, stream>>>(theta,
                                                                                           g);
    CK(cudaGetLastError());
    h->last_stream = stream;
    return BTDMA_OK;
}

int btdma_heat_step(btdma_heat_t h, double* theta, int n_steps, int use_graph,
                    cudaStream_t stream) {
    if (!h || !theta) return fail(BTDMA_ERR_ARG, "null argument");
    if (n_steps < 0) return fail(BTDMA_ERR_ARG, "n_steps must be >= 0");
    h->last_stream = stream;
    if (!use_graph) {
        for (int s = 0; s < n_steps; ++s) {
            const int rc = heat_enqueue(h, theta, stream);
            if (rc) return rc;
        }
        return BTDMA_OK;
    }
    if (!h->exec || h->graph_theta != theta) {
        if (h->exec) cudaGraphExecDestroy(h->exec);
        if (h->graph) cudaGraphDestroy(h->graph);
        h->exec = nullptr;
        h->graph = nullptr;
        // one uncaptured step on a zeroed scratch field first, so the kernels'
        // first-use attribute calls stay out of the capture (theta is untouched)
        const HeatGeom& g = h->g;
        CK(cudaMemsetAsync(h->scratch, 0, sizeof(double) * (size_t)(g.ix + 2) * (g.iy + 2) *
                                              (g.iz + 2), h->cap));
        int rc = heat_enqueue(h, h->scratch, h->cap);
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->cap));
        // capture on the private stream, after the caller's stream has reached
        // this point (the graph is launched on the caller's stream below)
        CK(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
        rc = heat_enqueue(h, theta, h->cap);
        cudaGraph_t gr = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->cap, &gr);
        if (rc) {
            if (gr) cudaGraphDestroy(gr);
            return rc;
        }
        CK(e);
        h->graph = gr;
        CK(cudaGraphInstantiate(&h->exec, gr, 0));
        h->graph_theta = theta;
    }
    for (int s = 0; s < n_steps; ++s) CK(cudaGraphLaunch(h->exec, stream));
    return BTDMA_OK;
}

int btdma_heat_step_profile(btdma_heat_t h, double* theta, double* times, cudaStream_t stream) {
    if (!h || !theta || !times) return fail(BTDMA_ERR_ARG, "null argument");
    const HeatGeom& g = h->g;
    cudaEvent_t ev[8];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    auto done = [&](int code) {
        for (auto& e : ev) cudaEventDestroy(e);
        return code;
    };
    const dim3 b1(128, 1, 1);
    const dim3 gr((g.ix + 127) / 128, g.iy, g.iz);
    const dim3 bt(HEAT_TILE, 8, 1);
    int rc = BTDMA_OK;
    cudaEventRecord(ev[0], stream);
    heat_rhs_z_kernel<<<gr, b1, 0, stream>>>(theta, h->buf0, g);
    cudaEventRecord(ev[1], stream);
    if ((rc = try_tile_const(h->buf0, h->buf0, g.ix * g.iy, g.iz, g.bz, true, h->status, stream, h->tab)) != 1)
        return done(rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "Z sweep not tileable"));
    cudaEventRecord(ev[2], stream);
    heat_z_to_y_kernel<<<gr, b1, 0, stream>>>(theta, h->buf0, h->buf1, g);
    cudaEventRecord(ev[3], stream);
    if ((rc = try_tile_const(h->buf1, h->buf1, g.ix * g.iz, g.iy, g.by, true, h->status, stream, h->tab)) != 1)
        return done(rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "Y sweep not tileable"));
    cudaEventRecord(ev[4], stream);
    heat_y_to_x_kernel<<<dim3((g.ix + HEAT_TILE - 1) / HEAT_TILE, (g.iy + HEAT_TILE - 1) / HEAT_TILE,
                              g.iz), bt, 0, stream>>>(theta, h->buf1, h->buf0, g);
    cudaEventRecord(ev[5], stream);
    if ((rc = try_tile_const(h->buf0, h->buf0, g.iy * g.iz, g.ix, g.bx, true, h->status, stream, h->tab)) != 1)
        return done(rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "X sweep not tileable"));
    cudaEventRecord(ev[6], stream);
    heat_update_kernel<<<dim3((g.iy + HEAT_TILE - 1) / HEAT_TILE, (g.ix + HEAT_TILE - 1) / HEAT_TILE,
                              g.iz), bt, 0, stream>>>(theta, h->buf0, g);
    cudaEventRecord(ev[7], stream);
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(ev[7]) != cudaSuccess)
        return done(fail(BTDMA_ERR_CUDA, "profiled heat step failed"));
    auto sec = [&](int a, int b) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[a], ev[b]);
        return 1e-3 * ms;
    };
    // the reference's 12 events (solve_theta.cu:436-439): rhs, solve_z, solve_y,
    // solve_x, etc, comm, tdma_{z,y,x}_comm, tdma_{z,y,x}_gpu
    const double t[12] = {sec(0, 1), sec(1, 3), sec(3, 5), sec(5, 7), 0.0, 0.0,
                          0.0,       0.0,       0.0,       sec(1, 2), sec(3, 4), sec(5, 6)};
    std::memcpy(times, t, sizeof t);
    h->last_stream = stream;
    return done(BTDMA_OK);
}

int btdma_heat_l2_error(btdma_heat_t h, const double* theta, double t_phys, double* l2) {
    if (!h || !theta || !l2) return fail(BTDMA_ERR_ARG, "null argument");
    const HeatGeom& g = h->g;
    const cudaStream_t st = h->last_stream;
    CK(cudaMemsetAsync(h->err, 0, sizeof(double), st));
    const double decay = exp(-3.0 * HEAT_PI * HEAT_PI * t_phys);
    heat_err_kernel<<<dim3((g.ix + 127) / 128, g.iy, g.iz), 128, 0, st>>>(theta, g, decay, h->err);
    CK(cudaGetLastError());
    double sum = 0.0;
    CK(cudaMemcpyAsync(&sum, h->err, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // normalised by (ix + 1)(iy + 1)(iz + 1), the reference's params.nx * ny * nz
    *l2 = sqrt(sum / ((double)(g.ix + 1) * (g.iy + 1) * (g.iz + 1)));
    return BTDMA_OK;
}

// -------------------------------------------- channel Poisson, wall-normal
struct btdma_poisson {
    int nz = 0, n_modes = 0, pin = 0;
    double* ga = nullptr;   // [nz] sub-diagonal per row
    double* gc = nullptr;   // [nz] super-diagonal per row
    double* lam = nullptr;  // [n_modes] kx^2 + ky^2 per mode
    unsigned* status = nullptr;
};

int btdma_poisson_create(int nz, const double* dz, const double* dmz, int n_modes,
                         const double* lambda, int pin_mode0, btdma_poisson_t* out) {
    if (!out) return fail(BTDMA_ERR_ARG, "null output handle");
    *out = nullptr;
    if (nz < 3 || n_modes <= 0 || !dz || !dmz || !lambda)
        return fail(BTDMA_ERR_ARG, "need nz >= 3, n_modes > 0 and the dz, dmz, lambda arrays");
    if (!tile_plan(nz, false, 8, 1).sys)
        return fail(BTDMA_ERR_UNSUPPORTED, "nz must be a multiple of 16 (tiled solve)");
    // row k: a = 1 / (dz[k+1] dmz[k+1]) (0 at the lower wall),
    //        c = 1 / (dz[k+1] dmz[k+2]) (0 at the upper wall)
    //   (k_build_poisson_tdma, PressureSolverGPU.cu:183-210)
    std::vector<double> ha(nz), hc(nz);
    for (int k = 0; k < nz; ++k) {
        ha[k] = k == 0 ? 0.0 : 1.0 / (dz[k + 1] * dmz[k + 1]);
        hc[k] = k == nz - 1 ? 0.0 : 1.0 / (dz[k + 1] * dmz[k + 2]);
    }
    btdma_poisson* h = new btdma_poisson();
    h->nz = nz;
    h->n_modes = n_modes;
    h->pin = pin_mode0 ? 1 : 0;
    auto cleanup = [&](int code) {
        btdma_poisson_destroy(h);
        return code;
    };
#define CKP(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return cleanup(fail(BTDMA_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_))); \
    } while (0)
    CKP(cudaMalloc(&h->ga, sizeof(double) * nz));
    CKP(cudaMalloc(&h->gc, sizeof(double) * nz));
    CKP(cudaMalloc(&h->lam, sizeof(double) * n_modes));
    CKP(cudaMalloc(&h->status, sizeof(unsigned)));
    CKP(cudaMemset(h->status, 0, sizeof(unsigned)));
    CKP(cudaMemcpy(h->ga, ha.data(), sizeof(double) * nz, cudaMemcpyHostToDevice));
    CKP(cudaMemcpy(h->gc, hc.data(), sizeof(double) * nz, cudaMemcpyHostToDevice));
    CKP(cudaMemcpy(h->lam, lambda, sizeof(double) * n_modes, cudaMemcpyHostToDevice));
#undef CKP
    *out = h;
    return BTDMA_OK;
}

int btdma_poisson_destroy(btdma_poisson_t h) {
    if (!h) return BTDMA_OK;
    cudaFree(h->ga);
    cudaFree(h->gc);
    cudaFree(h->lam);
    cudaFree(h->status);
    delete h;
    return BTDMA_OK;
}

int btdma_poisson_solve(btdma_poisson_t h, double* rhs, cudaStream_t stream) {
    if (!h || !rhs) return fail(BTDMA_ERR_ARG, "null argument");
    TileArgs g = {};
    g.ga = h->ga;
    g.gc = h->gc;
    g.glam = h->lam;
    g.gpin = h->pin;
    // complex rhs [nz][n_modes] = doubles [nz][2 n_modes]: real and imaginary
    // parts are systems 2m and 2m + 1 with one matrix
    const int rc = try_tile_gen<2>(rhs, rhs, 2 * h->n_modes, h->nz, g, h->status, stream);
    if (rc == 0)
        return fail(BTDMA_ERR_UNSUPPORTED, "rhs must be 16-byte aligned (tiled solve)");
    return rc < 0 ? rc : BTDMA_OK;
}

int btdma_poisson_status(btdma_poisson_t h, unsigned* status, cudaStream_t stream) {
    if (!h || !status) return fail(BTDMA_ERR_ARG, "null argument");
    CK(cudaMemcpyAsync(status, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    CK(cudaMemsetAsync(h->status, 0, sizeof(unsigned), stream));
    CK(cudaStreamSynchronize(stream));
    return BTDMA_OK;
}

// ------------------------------------------------ channel momentum ADI sweeps
struct btdma_momentum {
    MomGeom g{};
    int pbc[2] = {0, 0};
    double* tab = nullptr;  // [dir][comp][ta, tb, tc][n_dir rows]
    size_t tab_off[3][3] = {};
    double* buf = nullptr;  // nx * ny * nz, the sweep layout
    double* gtab = nullptr; // shared elimination factors of one sweep
    unsigned* status = nullptr;
};

int btdma_momentum_create(int nx, int ny, int nz, const double* dx0, const double* dmx0,
                          const double* dx1, const double* dmx1, const double* dx2,
                          const double* dmx2, int pbc_x, int pbc_y, btdma_momentum_t* out) {
    if (!out) return fail(BTDMA_ERR_ARG, "null output handle");
    *out = nullptr;
    if (nx <= 0 || ny <= 0 || nz <= 0 || !dx0 || !dmx0 || !dx1 || !dmx1 || !dx2 || !dmx2)
        return fail(BTDMA_ERR_ARG, "grid sizes and the six metric arrays are required");
    const int n[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d) {
        const bool cyc = d < 2 && (d == 0 ? pbc_x : pbc_y);
        if (!tile_plan(n[d], cyc, 8, 1).sys)
            return fail(BTDMA_ERR_UNSUPPORTED,
                        "sweep %d: n must be a multiple of 16 (n / 16 a power of two when "
                        "periodic)", d);
    }
    if ((long long)nx * ny * nz >= (1LL << 31))
        return fail(BTDMA_ERR_SIZE, "grid above 2^31 cells");
    // row tables (MomentumSolverGPU.cu:135-155, :176-180, :205-209): for row
    // r = 1..n, staggered when comp == dir;  a = -c ta, c = -c tc, b = 1 + c tb
    const double* dxs[3] = {dx0, dx1, dx2};
    const double* dms[3] = {dmx0, dmx1, dmx2};
    std::vector<double> tab;
    size_t off[3][3];
    for (int d = 0; d < 3; ++d)
        for (int comp = 0; comp < 3; ++comp) {
            off[d][comp] = tab.size();
            const int m = n[d];
            std::vector<double> ta(m), tb(m), tc(m);
            const double* dx = dxs[d];
            const double* dm = dms[d];
            for (int r = 1; r <= m; ++r) {
                const double ar = comp == d ? 1.0 / (dm[r] * dx[r - 1]) : 1.0 / (dx[r] * dm[r]);
                const double cr = comp == d ? 1.0 / (dm[r] * dx[r]) : 1.0 / (dx[r] * dm[r + 1]);
                double a_ = ar, b_ = ar + cr, c_ = cr;
                if (d == 2) {  // no-slip walls at both ends (one rank holds all of z)
                    const bool is_w = comp == 2;
                    if (r == 1) {
                        a_ = 0.0;
                        if (!is_w) b_ += ar;
                    }
                    if (r == m) {
                        c_ = 0.0;
                        if (!is_w) b_ += cr;
                    }
                    if (is_w && r == 1) a_ = b_ = c_ = 0.0;  // w = 0 on the wall
                }
                ta[r - 1] = a_;
                tb[r - 1] = b_;
                tc[r - 1] = c_;
            }
            tab.insert(tab.end(), ta.begin(), ta.end());
            tab.insert(tab.end(), tb.begin(), tb.end());
            tab.insert(tab.end(), tc.begin(), tc.end());
        }
    btdma_momentum* h = new btdma_momentum();
    h->g.nx = nx;
    h->g.ny = ny;
    h->g.nz = nz;
    h->pbc[0] = pbc_x ? 1 : 0;
    h->pbc[1] = pbc_y ? 1 : 0;
    std::memcpy(h->tab_off, off, sizeof off);
    auto cleanup = [&](int code) {
        btdma_momentum_destroy(h);
        return code;
    };
    if (cudaMalloc(&h->tab, sizeof(double) * tab.size()) != cudaSuccess ||
        cudaMemcpy(h->tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMalloc(&h->buf, sizeof(double) * (size_t)nx * ny * nz) != cudaSuccess ||
        cudaMalloc(&h->gtab, sizeof(double) * gen_table_doubles(std::max(nx, std::max(ny, nz)))) !=
            cudaSuccess ||
        cudaMalloc(&h->status, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(h->status, 0, sizeof(unsigned)) != cudaSuccess)
        return cleanup(fail(BTDMA_ERR_CUDA, "momentum buffers: %s",
                            cudaGetErrorString(cudaGetLastError())));
    *out = h;
    return BTDMA_OK;
}

int btdma_momentum_destroy(btdma_momentum_t h) {
    if (!h) return BTDMA_OK;
    cudaFree(h->tab);
    cudaFree(h->buf);
    cudaFree(h->gtab);
    cudaFree(h->status);
    delete h;
    return BTDMA_OK;
}

int btdma_momentum_sweep(btdma_momentum_t h, int dir, int comp, const double* q, double* dst,
                         double c, cudaStream_t stream) {
    if (!h || !q || !dst) return fail(BTDMA_ERR_ARG, "null argument");
    if (dir < 0 || dir > 2 || comp < 0 || comp > 2)
        return fail(BTDMA_ERR_ARG, "dir and comp must be 0, 1 or 2");
    const MomGeom& g = h->g;
    const int n[3] = {g.nx, g.ny, g.nz};
    const int n_sys = g.nx * g.ny * g.nz / n[dir];
    TileArgs t = {};
    t.cs = c;
    t.ga = h->tab + h->tab_off[dir][comp];
    t.gb = t.ga + n[dir];
    t.gc = t.gb + n[dir];
    const dim3 b1(128, 1, 1), bt(MOM_TILE, 8, 1);
    int rc;
    if (dir == 2) {
        mom_gather_kernel<2><<<dim3((g.nx + 127) / 128, g.ny, g.nz), b1, 0, stream>>>(
            q, h->buf, g, comp == 2 ? 1 : 0);
        CK(cudaGetLastError());
        rc = try_tile_gen<3, false>(h->buf, h->buf, n_sys, g.nz, t, h->status, stream, h->gtab);
    } else if (dir == 1) {
        mom_gather_kernel<1><<<dim3((g.nx + 127) / 128, g.nz, g.ny), b1, 0, stream>>>(q, h->buf,
                                                                                   g, 0);
        CK(cudaGetLastError());
        rc = h->pbc[1] ? try_tile_gen<3, true>(h->buf, h->buf, n_sys, g.ny, t, h->status, stream, h->gtab)
                       : try_tile_gen<3, false>(h->buf, h->buf, n_sys, g.ny, t, h->status, stream, h->gtab);
    } else {
        mom_gather_x_kernel<<<dim3((g.nx + MOM_TILE - 1) / MOM_TILE,
                                   (g.ny + MOM_TILE - 1) / MOM_TILE, g.nz), bt, 0, stream>>>(
            q, h->buf, g);
        CK(cudaGetLastError());
        rc = h->pbc[0] ? try_tile_gen<3, true>(h->buf, h->buf, n_sys, g.nx, t, h->status, stream, h->gtab)
                       : try_tile_gen<3, false>(h->buf, h->buf, n_sys, g.nx, t, h->status, stream, h->gtab);
    }
    if (rc != 1) return rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "sweep not tileable");
    if (dir == 2)
        mom_scatter_kernel<2><<<dim3((g.nx + 127) / 128, g.ny, g.nz), b1, 0, stream>>>(h->buf,
                                                                                     dst, g);
    else if (dir == 1)
        mom_scatter_kernel<1><<<dim3((g.nx + 127) / 128, g.nz, g.ny), b1, 0, stream>>>(h->buf,
                                                                                     dst, g);
    else
        mom_scatter_x_kernel<<<dim3((g.ny + MOM_TILE - 1) / MOM_TILE,
                                    (g.nx + MOM_TILE - 1) / MOM_TILE, g.nz), bt, 0, stream>>>(
            h->buf, dst, g);
    CK(cudaGetLastError());
    return BTDMA_OK;
}

int btdma_momentum_adi(btdma_momentum_t h, int comp, double* rhs, double* q_out, double c,
                       cudaStream_t stream) {
    int rc = btdma_momentum_sweep(h, 2, comp, rhs, rhs, c, stream);
    if (!rc) rc = btdma_momentum_sweep(h, 1, comp, rhs, rhs, c, stream);
    if (!rc) rc = btdma_momentum_sweep(h, 0, comp, rhs, q_out, c, stream);
    return rc;
}

int btdma_momentum_status(btdma_momentum_t h, unsigned* status, cudaStream_t stream) {
    if (!h || !status) return fail(BTDMA_ERR_ARG, "null argument");
    CK(cudaMemcpyAsync(status, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    CK(cudaMemsetAsync(h->status, 0, sizeof(unsigned), stream));
    CK(cudaStreamSynchronize(stream));
    return BTDMA_OK;
}

// ------------------------------------------------------------- self test
namespace {

// One thread waits, with the library's bounded wait, on an mbarrier that
// nothing ever arrives at: the wait must give up after `limit` polls and
// raise ST_TIMEOUT in the status word (the path every pipeline wait takes
// when a transfer never lands), leaving the context usable.
__global__ void selftest_wait_kernel(unsigned* status, uint32_t limit) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) (void)mbar_wait_bounded(&bar, 0, status, limit);
}

}  // namespace

int btdma_selftest_wait_timeout(int limit, unsigned* status_out, cudaStream_t stream) {
    if (limit <= 0 || limit > (1 << 16) || !status_out)
        return fail(BTDMA_ERR_ARG, "limit in [1, 65536] and an output word are required");
    unsigned* d = nullptr;
    CK(cudaMalloc(&d, sizeof(unsigned)));
    cudaMemsetAsync(d, 0, sizeof(unsigned), stream);
    selftest_wait_kernel<<<1, 32, 0, stream>>>(d, (uint32_t)limit);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(status_out, d, sizeof(unsigned),
                                              cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    CK(e);
    return BTDMA_OK;
}
