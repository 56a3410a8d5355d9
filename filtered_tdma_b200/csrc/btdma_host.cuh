// Host-side internals shared by the library's translation units: the solver
// handle, error reporting, tensor-map encoding and the launch planning of the
// tiled and segment kernels.  Not part of the C ABI (include/btdma.h).
#pragma once
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "btdma_common.cuh"
#include "k_segment.cuh"
#include "k_tile.cuh"
#include "k_tile_wide.cuh"

using namespace btdma;

// The tiled PaScaL solve of one uniform non-periodic batch [n_row][n_sys] with
// A, B, C, D of elem bytes (8: FP64, 4: FP32 storage), the kernel shape chosen
// as for a uniform batch (btdma_api.cu).  1: launched; 0: the shape is not
// tiled; < 0: error.
int tile_solve_batch(const void* A, const void* B, const void* C, const void* D, int elem,
                     double* X, int n_sys, int n_row, unsigned* status, cudaStream_t st);

struct btdma_handle {
    int method, P, precision, flags;
    int tile_shape = 0;  // BTDMA_TILE_AUTO / NARROW / WIDE (uniform PaScaL batches)
    int n_sys_cap, n_row_cap;
    double eps_constant;
    double* rho_row = nullptr;               // [n_row_cap] per-row spectral bound
    int* J = nullptr;                        // [P]
    unsigned long long* work = nullptr;      // [2P] J accumulators (kept zero between solves)
    unsigned* status = nullptr;              // device status word
    // Filtered: 1 when the latest solve took the exact reduced system (rho >= 0.5
    // or J >= m - 2 in a segment), set on the device by jfinal_kernel
    unsigned* exact = nullptr;
    bool last_filtered = false;              // the latest solve was a Filtered one (P > 1)
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
        // interleaved (non-periodic buckets): gathered into a row-interleaved
        // batch of npad x nbp systems, solved by the tiled kernel, scattered back;
        // ibuf holds the gathered A, B, C, D and the batch's x
        int inter = 0, npad = 0, nbp = 0;
        void* ibuf = nullptr;
    };
    std::vector<long long> rag_off;        // host copy of the offsets of the plan
    std::vector<unsigned char> rag_per;    // host copy of the periodic flags
    std::vector<RagBucket> rag_buckets;
    std::vector<int> rag_order;            // system ids, bucket by bucket
    long long* rag_d_off = nullptr;        // device offsets [n_sys + 1]
    int* rag_d_list = nullptr;             // device copy of rag_order
    int4* rag_d_tasks = nullptr;           // task tables [2 * n_sys]
    int4* rag_d_probe = nullptr;           // task table of one bucket being tuned [n_sys]
    int* rag_d_next = nullptr;             // task counters of the persistent launch [4]
    int rag_cls_first[3] = {}, rag_cls_count[3] = {};  // its classes (P = 256, 128, 64)
    int rag_warp_first = 0, rag_warp_count = 0;        // and its warp class
    bool rag_persist = false;              // CTA-kind buckets in the persistent launch
    // launches of a solve: warp-kind tasks (one launch), the long systems of
    // at most RAG_PERSIST_THREADS threads in one persistent launch (cta == 2),
    // longer ones per P (cta == 1)
    struct RagLaunch {
        int cta, P, first, count, mcap, staged;
    };
    std::vector<RagLaunch> rag_launches;
    static constexpr int RAG_STREAMS = 4;
    cudaStream_t rag_side[RAG_STREAMS] = {};
    cudaEvent_t rag_fork = nullptr, rag_join[RAG_STREAMS] = {};
    // host-buffer solves (btdma_solve_host): streams for copy-in, solve and
    // copy-out, and two device chunk buffers of A, B, C, D, X
    struct HostPipe {
        cudaStream_t s[3] = {};
        cudaEvent_t start = nullptr, done = nullptr;
        cudaEvent_t in[2] = {}, solved[2] = {}, out[2] = {};
        double* buf = nullptr;  // [2][5][chunk_elems]
        size_t chunk_elems = 0;
    };
    HostPipe* hp = nullptr;
};
namespace btdma_host {

extern thread_local std::string g_err;

// Records the message of a failing call (btdma_last_error) and returns code.
int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(BTDMA_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                              \
    } while (0)

// ------------------------------------------------------------ tensor maps
inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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
inline bool make_map(CUtensorMap* map, const void* ptr, int n_sys, int n_row) {
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

inline bool tma_ok(const void* p, int n_sys) {
    return ((reinterpret_cast<uintptr_t>(p) & 15) == 0) && (n_sys % 2 == 0);
}

inline int auto_segments(int n_row) {
    // ~64 rows per segment, at least 3, at most the cluster limit.
    if (n_row < 6) return 1;
    int P = (n_row + 63) / 64;
    P = std::max(2, std::min(P, SEG_MAX_P));
    while (P > 1 && n_row / P < 3) --P;
    return P;
}

inline int seg_mcap(int n_row, int P) {
    int mmax = (n_row + P - 1) / P;
    return (mmax + SEG_BOXR - 1) / SEG_BOXR * SEG_BOXR;
}

inline int max_smem_optin() {
    static int v = -1;
    if (v < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
            v = 48 * 1024;
    }
    return v;
}

template <int METHOD, bool CYCLIC, int RR>
int launch_seg_rr(const CUtensorMap* maps, const SegArgs& a, int groups, cudaStream_t st) {
    auto kern = seg_f64_kernel<METHOD, CYCLIC, RR>;
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
    cfg.dynamicSmemBytes = seg_smem_bytes(a.mcap, a.P, CYCLIC, METHOD == SEG_PASCAL, RR);
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

// SEG_REG leading rows of each segment go to registers when every segment has
// room for them (seg_reg_rows).
template <int METHOD, bool CYCLIC>
int launch_seg(const CUtensorMap* maps, const SegArgs& a, int groups, cudaStream_t st) {
    if (seg_reg_rows(a.n_row, a.P) == SEG_REG)
        return launch_seg_rr<METHOD, CYCLIC, SEG_REG>(maps, a, groups, st);
    return launch_seg_rr<METHOD, CYCLIC, 0>(maps, a, groups, st);
}

// 3-D view [nseg][TILE_MT][n_sys] of an [n_row x n_sys] FP64 array; boxes of
// tile_rps(elem, na) rows of `nsc` consecutive sub-segments for `sys` systems
// (na: arrays of the ring the boxes go to).
inline bool make_tile_map(CUtensorMap* map, const void* ptr, int n_sys, int nseg, int sys,
                          int nsc, int elem = 8, int na = 4) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {(cuuint64_t)n_sys, (cuuint64_t)TILE_MT, (cuuint64_t)nseg};
    cuuint64_t strides[2] = {(cuuint64_t)n_sys * elem, (cuuint64_t)n_sys * TILE_MT * elem};
    cuuint32_t box[3] = {(cuuint32_t)sys, (cuuint32_t)tile_rps(elem, na), (cuuint32_t)nsc};
    cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType dt =
        elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUresult r = fn(map, dt, 3, const_cast<void*>(ptr), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

inline int num_sms() {
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
    int pr = 1;  // sub-segments per thread (2: shared-matrix sweeps of 18..32 sub-segments)
};

inline int max_smem_per_sm() {
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
// sh: shared-matrix sweep (factor table and lane table in shared memory).
// tstore: the sweep stores rows contiguously through a shared tile (xrs == 1).
inline TilePlan tile_plan(int n_row, bool cyclic, int elem = 8, int na = 4, bool sh = false,
                          bool tstore = false) {
    TilePlan pl;
    if (n_row % TILE_MT != 0) return pl;
    const int nseg = n_row / TILE_MT;
    if (cyclic && (nseg & (nseg - 1)) != 0) return pl;  // periodic PCR needs 2^k rows
    int sys, cl = 0, pr = 1;
    if (sh && nseg > 16 && nseg <= 32 && nseg % 2 == 0) {
        // Longer shared-matrix sweeps: two sub-segments per thread, so a CTA of
        // 16 systems has at most 256 threads and two share an SM, as for the
        // shorter sweeps below.
        sys = 16;
        cl = 1;
        pr = 2;
    } else if (sh && nseg <= 16) {
        // Shared-matrix sweeps of up to 16 sub-segments: CTAs of at most
        // TILE_SH_THREADS threads, two or more per SM, so that one CTA's reduced
        // solve overlaps another's sweeps.  (Longer systems keep one CTA of up
        // to 512 threads: splitting them over a 2-CTA cluster was measured
        // slower, the cluster barriers waiting for the partner CTA.)
        sys = std::min(128, TILE_SH_THREADS / tile_lanes(nseg));
        cl = 1;
    } else if (nseg <= 4) {
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
    size_t cap = (size_t)max_smem_optin();
    if (sh) {  // an equal share of the SM per resident CTA (128 registers a thread)
        const int per_sm = std::max(1, 65536 / (sys * (nseg / cl / pr) * 128));
        cap = std::min(cap, (size_t)max_smem_per_sm() / per_sm - 1024);
    }
    while (nst >= 3 && tile_smem_bytes(sys, nseg / cl, nseg, sys / cl, nst, elem, na, sh, 0,
                                       tstore && cl == 1 ? n_row / pr : 0) > cap)
        --nst;
    if (nst < 3) return pl;
    pl.sys = sys;
    pl.cl = cl;
    pl.nst = nst;
    pl.nseg = nseg;
    pl.pr = pr;
    return pl;
}

template <int SYS, bool CYCLIC, typename TIN = double, typename TC = double, int GEN = 0,
          int PR = 1, bool FILT = false>
int launch_tile_sys(const CUtensorMap* maps, const TileArgs& a, cudaStream_t st) {
    auto kern = tile_f64_kernel<SYS, CYCLIC, TIN, TC, GEN, PR, FILT>;
    static bool attr_done = false;
    if (!attr_done) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                max_smem_optin()));
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        attr_done = true;
    }
    const int threads = SYS * a.nseg / a.cl / PR;
    if (PR > 1 && (a.nseg > 32 || a.cl != 1 || (a.nseg / a.cl) % PR != 0))
        return fail(BTDMA_ERR_UNSUPPORTED, "%d sub-segments per thread need one CTA of <= 32",
                    PR);
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(threads, 1, 1);
    constexpr bool SHT = GEN == 1 || GEN == 3 || GEN == 4 || GEN == 5;
    // the kernel stages row-contiguous stores (xrs == 1) in a tile after the mbarriers
    const bool tstore = SHT && a.xblk > 0 && a.xrs == 1 && a.cl == 1;
    cfg.dynamicSmemBytes = tile_smem_bytes(SYS, a.nseg / a.cl, a.nseg, SYS / a.cl, a.nst,
                                           (int)sizeof(TIN), GEN ? 1 : 4, SHT, GEN,
                                           tstore ? a.n_row / PR : 0);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = num_sms();
    if (a.cl == 1) {  // as many CTAs as fit on an SM (several for shared-matrix sweeps)
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

template <typename TIN, typename TC, bool FILT = false>
int launch_tile_plan(const TilePlan& pl, const CUtensorMap* maps, const TileArgs& a, bool cyclic,
                     cudaStream_t st) {
    switch (pl.sys * 2 + (cyclic ? 1 : 0)) {
        case 256: return launch_tile_sys<128, false, TIN, TC, 0, 1, FILT>(maps, a, st);
        case 257: return launch_tile_sys<128, true, TIN, TC, 0, 1, FILT>(maps, a, st);
        case 128: return launch_tile_sys<64, false, TIN, TC, 0, 1, FILT>(maps, a, st);
        case 129: return launch_tile_sys<64, true, TIN, TC, 0, 1, FILT>(maps, a, st);
        case 64: return launch_tile_sys<32, false, TIN, TC, 0, 1, FILT>(maps, a, st);
        case 65: return launch_tile_sys<32, true, TIN, TC, 0, 1, FILT>(maps, a, st);
        case 33: return launch_tile_sys<16, true, TIN, TC, 0, 1, FILT>(maps, a, st);
        default: return launch_tile_sys<16, false, TIN, TC, 0, 1, FILT>(maps, a, st);
    }
}

// BTDMA_TILE_AUTO's choice between the kernels for a shape both take, from
// B200 measurements (262144 x 512, 524288 x 256, 1048576 x 128; ms):
//   FP32 storage  narrow 1.03 / 0.81 / 0.83   wide 0.82 / 0.73 / 0.72
//   FP64          narrow 1.06 / 0.97 / 0.96   wide 1.03 / 1.02 / 1.01
// The narrow kernel reads 64-byte row pieces for FP32 at 512 rows and 128-byte
// pieces elsewhere; the wide kernel's extra pass over half the rows pays off
// for FP32 storage everywhere and for FP64 above 16 sub-segments only.
inline bool wide_by_default(int n_row, int elem) {
    return elem == 4 || n_row / TILE_MT > 16;
}

// Plan of the wide-box kernel (k_tile_wide.cuh): sys == 0 when the shape does
// not take it.
inline TilePlan tile_wide_plan(int n_row, bool cyclic, int elem) {
    TilePlan pl;
    if (n_row % TILE_MT != 0) return pl;
    const int nseg = n_row / TILE_MT;
    if (nseg < 8 || nseg > 32 || nseg % 2 != 0) return pl;
    if (cyclic && (nseg & (nseg - 1)) != 0) return pl;
    const int h = nseg / 2;
    const int sys = h > 8 ? 32 : (h > 4 ? 64 : 128);
    int nst = TILE_MAX_NST;
    while (nst >= 3 && tile_wide_smem_bytes(sys, nseg, nst, elem) > (size_t)max_smem_optin())
        --nst;
    if (nst < 3) return pl;
    pl.sys = sys;
    pl.cl = 1;
    pl.nst = nst;
    pl.nseg = nseg;
    return pl;
}

template <int SYS, bool CYCLIC, typename TIN, bool FILT = false>
int launch_tile_wide(const CUtensorMap* maps, const TileArgs& a, cudaStream_t st) {
    auto kern = tile_wide_kernel<SYS, CYCLIC, TIN, FILT>;
    static bool attr_done = false;
    if (!attr_done) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                max_smem_optin()));
        attr_done = true;
    }
    const int threads = SYS * (a.nseg / 2);
    const size_t smem = tile_wide_smem_bytes(SYS, a.nseg, a.nst, (int)sizeof(TIN));
    const int grid = std::min(num_sms(), a.n_groups);
    kern<<<grid, threads, smem, st>>>(maps[0], maps[1], maps[2], maps[3], a);
    CK(cudaGetLastError());
    return BTDMA_OK;
}

template <typename TIN, bool FILT = false>
int launch_tile_wide_plan(const TilePlan& pl, const CUtensorMap* maps, const TileArgs& a,
                          bool cyclic, cudaStream_t st) {
    switch (pl.sys * 2 + (cyclic ? 1 : 0)) {
        case 256: return launch_tile_wide<128, false, TIN, FILT>(maps, a, st);
        case 257: return launch_tile_wide<128, true, TIN, FILT>(maps, a, st);
        case 128: return launch_tile_wide<64, false, TIN, FILT>(maps, a, st);
        case 129: return launch_tile_wide<64, true, TIN, FILT>(maps, a, st);
        case 65: return launch_tile_wide<32, true, TIN, FILT>(maps, a, st);
        default: return launch_tile_wide<32, false, TIN, FILT>(maps, a, st);
    }
}

inline bool tma_ok_elem(const void* p, int n_sys, int elem) {
    return ((reinterpret_cast<uintptr_t>(p) & 15) == 0) && ((size_t)n_sys * elem) % 16 == 0;
}

// Returns 1 when the tiled kernel was launched, 0 when the shape needs the
// cluster-per-segment kernel, < 0 on error.
// TC: arithmetic of the local sweeps; accumulate: X += solution; gate: the
// kernel does nothing while *gate == 0 (gate_zero: while *gate != 0); filt_r >
// 0: Filtered's reduced system with segments of filt_r sub-segments.
// shape: BTDMA_TILE_* (the wide-box kernel serves FP64-arithmetic solves that
// do not accumulate).
template <typename TIN, typename TC = double>
int try_tile(const TIN* A, const TIN* B, const TIN* C, const TIN* D, double* X, int n_sys,
             int n_row, bool cyclic, unsigned* status, cudaStream_t st, bool accumulate = false,
             const unsigned* gate = nullptr, int shape = BTDMA_TILE_NARROW, int filt_r = 0,
             bool gate_zero = false) {
    const int elem = (int)sizeof(TIN);
    bool wide = false;
    TilePlan pl;
    if (shape != BTDMA_TILE_NARROW && sizeof(TC) == 8 && !accumulate) {
        pl = tile_wide_plan(n_row, cyclic, elem);
        wide = pl.sys != 0 && (shape == BTDMA_TILE_WIDE || wide_by_default(n_row, elem));
    }
    if (!wide) {
        pl = tile_plan(n_row, cyclic, elem);
        // small batches: fewer systems per CTA until every SM has a group (the
        // ring's stages only get smaller, so its depth stays valid)
        while (pl.sys > 16 && pl.cl == 1 && (n_sys + pl.sys - 1) / pl.sys < num_sms())
            pl.sys >>= 1;
    }
    if (pl.sys == 0) return 0;
    if (!(tma_ok_elem(A, n_sys, elem) && tma_ok_elem(B, n_sys, elem) &&
          tma_ok_elem(C, n_sys, elem) && tma_ok_elem(D, n_sys, elem)))
        return 0;
    // sub-segments per TMA box: the CTA's share (narrow), or half a system (wide)
    const int nsc = wide ? pl.nseg / 2 : pl.nseg / pl.cl;
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
    a.mode = (accumulate ? TILE_MODE_ACCUMULATE : 0) | (gate_zero ? TILE_MODE_GATE_ZERO : 0) |
             (filt_r << TILE_MODE_FILT_SHIFT);
    a.gate = gate;
    a.status = status;
    int rc;
    if constexpr (std::is_same<TIN, double>::value && std::is_same<TC, double>::value) {
        if (filt_r > 0) {  // Filtered's instantiations (FP64 only)
            rc = wide ? launch_tile_wide_plan<TIN, true>(pl, maps, a, cyclic, st)
                      : launch_tile_plan<TIN, TC, true>(pl, maps, a, cyclic, st);
            return rc == BTDMA_OK ? 1 : rc;
        }
    } else {
        if (filt_r > 0) return fail(BTDMA_ERR_UNSUPPORTED, "Filtered tiles are FP64 only");
    }
    rc = wide ? launch_tile_wide_plan<TIN>(pl, maps, a, cyclic, st)
              : launch_tile_plan<TIN, TC>(pl, maps, a, cyclic, st);
    return rc == BTDMA_OK ? 1 : rc;
}

// Factor table of a shared-matrix sweep (GEN 1 or 3) of n_row rows: the
// elimination of every sub-segment and the reduced system's lane table, built
// by one small launch.  It depends only on the matrix (gen's coefficient
// fields), so a caller whose matrix does not change builds it once.
template <int GEN, bool CYC = false>
int build_gen_table(int n_row, const TileArgs& gen, double* tab, cudaStream_t st) {
    static_assert(GEN == 1 || GEN == 3, "shared-matrix modes only");
    const TilePlan pl = tile_plan(n_row, CYC, 8, 1, true);
    if (pl.sys == 0) return fail(BTDMA_ERR_UNSUPPORTED, "%d rows are not tileable", n_row);
    if (!tab) return fail(BTDMA_ERR_ARG, "shared-matrix sweep without a factor table");
    TileArgs a = gen;
    a.n_row = n_row;
    a.nseg = pl.nseg;
    a.cl = pl.cl;
    a.nst = pl.nst;
    tile_table_kernel<GEN, CYC><<<(pl.nseg + 127) / 128, 128, 0, st>>>(a, tab);
    CK(cudaGetLastError());
    return BTDMA_OK;
}

// Generated-coefficient batch, only D read (the GEN modes of the tiled
// kernel; the coefficient fields of `gen` are used, the rest is filled here).
// Returns 1 when launched, 0 when the shape is not tiled, < 0 on error.
// GEN 1 and 3 (one matrix for every system): `tab` is device scratch of
// gen_table_doubles(n_row) doubles for the shared elimination factors, built
// here unless `table_ready` (built earlier by build_gen_table for this matrix).
template <int GEN, bool CYC = false>
int try_tile_gen(const double* D, double* X, int n_sys, int n_row, const TileArgs& gen,
                 unsigned* status, cudaStream_t st, double* tab = nullptr,
                 bool table_ready = false) {
    const bool tstore = (GEN == 1 || GEN == 3) && gen.xblk > 0 && gen.xrs == 1;
    const TilePlan pl = tile_plan(n_row, CYC, 8, 1, GEN == 1 || GEN == 3, tstore);
    if (pl.sys == 0 || !tma_ok_elem(D, n_sys, 8)) return 0;
    const int nsc = pl.nseg / pl.cl;
    CUtensorMap maps[4];
    if (!make_tile_map(&maps[3], D, n_sys, pl.nseg, pl.sys, nsc, 8, 1)) return 0;
    maps[0] = maps[1] = maps[2] = maps[3];  // not read in this mode
    TileArgs a = gen;
    a.X = X;
    a.n_sys = n_sys;
    a.n_row = n_row;
    a.nseg = pl.nseg;
    a.cl = pl.cl;
    a.nst = pl.nst;
    a.n_groups = (n_sys + pl.sys - 1) / pl.sys;
    a.status = status;  // the layout map (xblk ...) comes with gen
    if constexpr (GEN == 1 || GEN == 3) {
        if (!tab) return fail(BTDMA_ERR_ARG, "shared-matrix sweep without a factor table");
        if (!table_ready) {
            tile_table_kernel<GEN, CYC><<<(pl.nseg + 127) / 128, 128, 0, st>>>(a, tab);
            CK(cudaGetLastError());
        }
        a.gtab = tab;
    }
    int rc;
    if constexpr (GEN == 1 || GEN == 3) {
        if (pl.pr == 2) {
            rc = launch_tile_sys<16, CYC, double, double, GEN, 2>(maps, a, st);
            return rc == BTDMA_OK ? 1 : rc;
        }
    }
    switch (pl.sys) {
        case 128: rc = launch_tile_sys<128, CYC, double, double, GEN>(maps, a, st); break;
        case 64: rc = launch_tile_sys<64, CYC, double, double, GEN>(maps, a, st); break;
        case 32: rc = launch_tile_sys<32, CYC, double, double, GEN>(maps, a, st); break;
        default: rc = launch_tile_sys<16, CYC, double, double, GEN>(maps, a, st); break;
    }
    return rc == BTDMA_OK ? 1 : rc;
}

// Heat Z sweep with the right-hand side fused (GEN 4 of the tiled kernel):
// the plan (16 systems per group, one CTA of 16 x n_row / 16 threads, 2 to 32
// sub-segments), or sys == 0 when the shape does not take it.
inline TilePlan tile_plan_heat_z(int n_row) {
    TilePlan pl;
    if (n_row % TILE_MT != 0) return pl;
    const int nseg = n_row / TILE_MT;
    if (nseg < 2 || nseg > 32) return pl;
    // one sub-segment per thread: with two, the stencil's stage values and the
    // two recurrences exceed 128 registers and spill
    const int pr = 1;
    const int T = TILE_HEAT_SYS * nseg / pr;
    const int per_sm = std::max(1, 65536 / (T * 128));
    const size_t cap = std::min((size_t)max_smem_optin(), (size_t)max_smem_per_sm() / per_sm - 1024);
    int nst = TILE_MAX_NST_CONST;
    while (nst >= 2 &&
           tile_smem_bytes(TILE_HEAT_SYS, nseg, nseg, TILE_HEAT_SYS, nst, 8, 1, true, 4) > cap)
        --nst;
    if (nst < 2) return pl;
    pl.sys = TILE_HEAT_SYS;
    pl.cl = 1;
    pl.nst = nst;
    pl.nseg = nseg;
    pl.pr = pr;
    return pl;
}

// 4-D view of the heat field theta [(iz + 2) x (iy + 2) x (ix + 2)] for the
// fused Z sweep: (x = i, y = j, row within the sub-segment, sub-segment) from
// plane k = 1; boxes of TILE_HEAT_BOX_I x 3 x 4 rows x nsc sub-segments.
inline bool make_heat_theta_map(CUtensorMap* map, const double* theta, int ix, int iy, int nseg,
                                int nsc) {
    auto fn = encode_fn();
    if (!fn) return false;
    const size_t nx = (size_t)ix + 2, plane = nx * ((size_t)iy + 2);
    cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)iy + 2, (cuuint64_t)TILE_MT,
                          (cuuint64_t)nseg};
    cuuint64_t strides[3] = {nx * sizeof(double), plane * sizeof(double),
                             (cuuint64_t)TILE_MT * plane * sizeof(double)};
    cuuint32_t box[4] = {(cuuint32_t)TILE_HEAT_BOX_I, 3u, (cuuint32_t)tile_rps(8, 1),
                         (cuuint32_t)nsc};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(theta + plane),
                    dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// The heat Z sweep with its right-hand side computed inside the solve from
// theta (GEN 4).  gen carries the sweep's fields: cs = bz, cbound = 1, ga / gb
// / gc = cos(pi x), cos(pi y), cos(pi z) tables (ghosts included), glam = the
// device array {bx, by, dt 3 pi^2, iy, iz}, xblk = ix and the output layout map.
// tab: the Z matrix's factor table (build_gen_table<1>).  Returns 1 when
// launched, 0 when the shape is not taken, < 0 on error.
inline int try_heat_z(const double* theta, double* X, int ix, int iy, int iz, const TileArgs& gen,
                      unsigned* status, cudaStream_t st, const double* tab) {
    const TilePlan pl = tile_plan_heat_z(iz);
    if (pl.sys == 0 || ix % TILE_HEAT_SYS != 0 ||
        (reinterpret_cast<uintptr_t>(theta) & 15) != 0 || ((size_t)(ix + 2) * 8) % 16 != 0)
        return 0;
    CUtensorMap maps[4];
    if (!make_heat_theta_map(&maps[3], theta, ix, iy, pl.nseg, pl.nseg)) return 0;
    maps[0] = maps[1] = maps[2] = maps[3];  // not read in this mode
    TileArgs a = gen;
    a.X = X;
    a.n_sys = ix * iy;
    a.n_row = iz;
    a.nseg = pl.nseg;
    a.cl = pl.cl;
    a.nst = pl.nst;
    a.n_groups = a.n_sys / TILE_HEAT_SYS;
    a.status = status;
    a.gtab = tab;
    const int rc = launch_tile_sys<TILE_HEAT_SYS, false, double, double, 4>(maps, a, st);
    return rc == BTDMA_OK ? 1 : rc;
}

// Momentum z sweep reading the ghosted field directly (GEN 5 of the tiled
// kernel): 16 systems per group, two sub-segments per thread above 16
// sub-segments (as tile_plan's shared-matrix sweeps), or sys == 0.
inline TilePlan tile_plan_field_z(int n_row) {
    TilePlan pl;
    if (n_row % TILE_MT != 0) return pl;
    const int nseg = n_row / TILE_MT;
    if (nseg < 2 || nseg > 32) return pl;
    const int pr = nseg > 16 && nseg % 2 == 0 ? 2 : 1;
    const int T = TILE_HEAT_SYS * nseg / pr;
    const int per_sm = std::max(1, 65536 / (T * 128));
    const size_t cap = std::min((size_t)max_smem_optin(), (size_t)max_smem_per_sm() / per_sm - 1024);
    int nst = TILE_MAX_NST_CONST;
    while (nst >= 3 &&
           tile_smem_bytes(TILE_HEAT_SYS, nseg, nseg, TILE_HEAT_SYS, nst, 8, 1, true, 5) > cap)
        --nst;
    if (nst < 3) return pl;
    pl.sys = TILE_HEAT_SYS;
    pl.cl = 1;
    pl.nst = nst;
    pl.nseg = nseg;
    pl.pr = pr;
    return pl;
}

// 4-D view of a ghosted field q [(nz + 2) x (ny + 2) x (nx + 2)] for the z
// sweep: (x = i, y = j, row within the sub-segment, sub-segment) from plane
// k = 1; boxes of TILE_HEAT_BOX_I x 1 x 4 rows x nsc sub-segments.
inline bool make_field_row_map(CUtensorMap* map, const double* q, int nx, int ny, int nseg,
                               int nsc) {
    auto fn = encode_fn();
    if (!fn) return false;
    const size_t rx = (size_t)nx + 2, plane = rx * ((size_t)ny + 2);
    cuuint64_t dims[4] = {(cuuint64_t)rx, (cuuint64_t)ny + 2, (cuuint64_t)TILE_MT,
                          (cuuint64_t)nseg};
    cuuint64_t strides[3] = {rx * sizeof(double), plane * sizeof(double),
                             (cuuint64_t)TILE_MT * plane * sizeof(double)};
    cuuint32_t box[4] = {(cuuint32_t)TILE_HEAT_BOX_I, 1u, (cuuint32_t)tile_rps(8, 1),
                         (cuuint32_t)nsc};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(q + plane), dims,
                    strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// The momentum z sweep straight from the ghosted field q (no gather): system
// s = (j - 1) nx + (i - 1), row k - 1; x through gen's layout map (xblk = nx).
// gen carries the GEN 3 row tables (ga, gb, gc), cs and the map; pin: row 0 is
// x = 0 (the w component).  tab: the (z, comp) factor table, built here unless
// table_ready.  Returns 1 when launched, 0 when the shape is not taken, < 0 on
// error.
inline int try_mom_z(const double* q, double* X, int nx, int ny, int nz, const TileArgs& gen,
                     int pin, unsigned* status, cudaStream_t st, double* tab, bool table_ready) {
    const TilePlan pl = tile_plan_field_z(nz);
    if (pl.sys == 0 || nx % TILE_HEAT_SYS != 0 || (reinterpret_cast<uintptr_t>(q) & 15) != 0 ||
        ((size_t)(nx + 2) * 8) % 16 != 0 || gen.xblk != nx)
        return 0;
    CUtensorMap maps[4];
    if (!make_field_row_map(&maps[3], q, nx, ny, pl.nseg, pl.nseg)) return 0;
    maps[0] = maps[1] = maps[2] = maps[3];  // not read in this mode
    TileArgs a = gen;
    a.X = X;
    a.n_sys = nx * ny;
    a.n_row = nz;
    a.nseg = pl.nseg;
    a.cl = pl.cl;
    a.nst = pl.nst;
    a.n_groups = a.n_sys / TILE_HEAT_SYS;
    a.status = status;
    a.gpin = pin;
    if (!table_ready) {
        tile_table_kernel<3, false><<<(pl.nseg + 127) / 128, 128, 0, st>>>(a, tab);
        CK(cudaGetLastError());
    }
    a.gtab = tab;
    const int rc = pl.pr == 2
                       ? launch_tile_sys<TILE_HEAT_SYS, false, double, double, 5, 2>(maps, a, st)
                       : launch_tile_sys<TILE_HEAT_SYS, false, double, double, 5>(maps, a, st);
    return rc == BTDMA_OK ? 1 : rc;
}

template <bool CYCLIC>
int launch_seg_method(int method, const CUtensorMap* maps, const SegArgs& a, int groups,
                      cudaStream_t st) {
    switch (method) {
        case BTDMA_PASCAL: return launch_seg<SEG_PASCAL, CYCLIC>(maps, a, groups, st);
        case BTDMA_FILTERED_V1: return launch_seg<SEG_FILT_V1, CYCLIC>(maps, a, groups, st);
        default: return launch_seg<SEG_FILT_V2, CYCLIC>(maps, a, groups, st);
    }
}

}  // namespace btdma_host

using namespace btdma_host;
