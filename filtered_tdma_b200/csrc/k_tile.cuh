// Register-tiled segmented solve: the fast exact path (PaScaL, P >= 2).
//
// Every system is cut into NSEG sub-segments of TILE_MT = 16 rows; one thread
// owns one sub-segment of one system and keeps its whole elimination state in
// registers.  A persistent CTA of SYS systems x NSEG sub-segments (<= 512
// threads) walks over groups of SYS systems:
//
//   1. Forward pass (one row of every sub-segment per step).  Row k of all NSEG
//      sub-segments of SYS systems arrives in one TMA box of a 3-D view
//      [NSEG][TILE_MT][n_sys] of each array, through a TILE_NST-stage shared
//      memory ring (an mbarrier per stage); the last warp to finish reading a
//      stage refills it, so the ring stays TILE_NST rows ahead of the slowest
//      warp and the next group's first rows are in flight while this group
//      finishes.  Each
//      thread runs the modified Thomas elimination of PaScaL
//      (libs/pascal_tdma/cpu/pascal_tdma.cpp:131-170) on its 16 rows:
//          alpha_k x_first + x_k + gamma_k x_{k+1} = delta_k,
//      and, instead of a second (backward) sweep, accumulates the reduced first
//      row in running products:  with pi_1 = 1, pi_{k+1} = -gamma_k pi_k,
//          delta''_1 = sum_{k=1}^{M-2} pi_k delta_k,  alpha''_1 = sum pi_k alpha_k,
//          gamma''_1 = -pi_{M-1},
//      which is the backward recurrence of pascal_tdma.cpp:157-170 evaluated
//      at row 1, followed by the row-0 reduction of pascal_tdma.cpp:173-178.
//   2. Reduced system: rows (2q, 2q+1) = first/last row of sub-segment q, unit
//      diagonal, solved by parallel cyclic reduction in shared memory
//      (log2(2 NSEG) steps, one barrier each) instead of the reference's
//      all-to-all transpose + serial Thomas (pascal_tdma.cpp:185-210).
//   3. Back substitution from registers:  x_k = delta_k - alpha_k x_first -
//      gamma_k x_{k+1}, k = M-2..1, and x is stored (coalesced, SYS systems wide).
//
// HBM traffic: A, B, C, D read once (32 B/row), x written once (8 B/row).
// The result equals the serial Thomas solution to rounding (<= 1e-12 relative
// on the tested batches), not bit for bit: the operation order differs from the
// reference's.  Needs n_row = 16 * NSEG with NSEG <= 32, even n_sys and 16-byte
// aligned arrays (TMA); periodic systems need NSEG to be a power of two.
#pragma once

#include "btdma_common.cuh"

namespace btdma {

constexpr int TILE_MT = 16;       // rows per sub-segment (per thread)
constexpr int TILE_NST = 10;      // TMA ring stages
constexpr int TILE_MAX_THREADS = 512;

struct TileArgs {
    double* X;
    int n_sys, n_row, nseg, n_groups;
    int cyclic;
    unsigned* status;
};

// PCR buffers: [2 buffers][3 fields l,u,r][N + 2 rows][SYS], rows -1 and N are
// zero guard rows so that out-of-range neighbours need no branch.
__host__ __device__ __forceinline__ size_t tile_pcr_doubles(int threads, int sys) {
    return 2ull * 3 * (2 * threads + 2 * sys);
}
__host__ __device__ __forceinline__ size_t tile_smem_bytes(int threads, int sys) {
    size_t ring = (size_t)TILE_NST * 4 * threads * sizeof(double);
    size_t pcr = tile_pcr_doubles(threads, sys) * sizeof(double);
    size_t bars = TILE_NST * (sizeof(uint64_t) + sizeof(int));
    return ring + pcr + bars + 128;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 3-D tiled load (x = system, y = row inside the sub-segment, z = sub-segment).
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

template <int SYS, bool CYCLIC>
__global__ void __launch_bounds__(TILE_MAX_THREADS, 1)
tile_f64_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmD,
                const TileArgs args) {
    constexpr int M = TILE_MT;
    extern __shared__ unsigned char smem_raw[];
    const int nseg = args.nseg;
    const int T = SYS * nseg;  // == blockDim.x
    const int N = 2 * nseg;    // reduced rows per system
    double* ring = reinterpret_cast<double*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    double* pcr = ring + (size_t)TILE_NST * 4 * T;
    uint64_t* full = reinterpret_cast<uint64_t*>(pcr + tile_pcr_doubles(T, SYS));
    int* readers = reinterpret_cast<int*>(full + TILE_NST);  // warps done with a slot

    const int tid = threadIdx.x;
    const int s = tid % SYS;
    const int q = tid / SYS;
    const size_t ns = (size_t)args.n_sys;
    const int nwarps = (T + 31) / 32;

    // PCR field bases for this thread's system column; row r lives at [r * SYS]
    // from base + SYS (row -1 is the first guard row).
    const int fs = (N + 2) * SYS;       // field stride
    double* const pb = pcr + SYS + s;   // buffer 0, field l, row 0
    auto FB = [&](int b, int f) { return pb + (b * 3 + f) * fs; };

    if (tid == 0) {
        for (int i = 0; i < TILE_NST; ++i) {
            mbar_init(&full[i], 1);
            readers[i] = 0;
        }
        fence_mbar_init();
    }
    if (tid < SYS) {  // zero guard rows (never written again)
        for (int bf = 0; bf < 6; ++bf) {
            pb[bf * fs - SYS] = 0.0;
            pb[bf * fs + N * SYS] = 0.0;
        }
    }
    __syncthreads();

    const int n_my = args.n_groups > (int)blockIdx.x
                         ? (args.n_groups - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x
                         : 0;
    const int total = n_my * M;  // ring stages this CTA consumes
    const uint32_t stage_bytes = 4u * T * sizeof(double);

    auto issue = [&](int t) {  // one thread
        const int slot = t % TILE_NST;
        const int g = (int)blockIdx.x + (t / M) * (int)gridDim.x;
        const int k = t % M;
        double* dst = ring + (size_t)slot * 4 * T;
        mbar_expect_tx(&full[slot], stage_bytes);
        tma_load_3d(dst + 0 * T, &tmA, g * SYS, k, 0, &full[slot]);
        tma_load_3d(dst + 1 * T, &tmB, g * SYS, k, 0, &full[slot]);
        tma_load_3d(dst + 2 * T, &tmC, g * SYS, k, 0, &full[slot]);
        tma_load_3d(dst + 3 * T, &tmD, g * SYS, k, 0, &full[slot]);
    };
    bool ok = true;
    if (tid == 0)
        for (int t = 0; t < TILE_NST && t < total; ++t) issue(t);

    bool finite = true;
    int slot = 0;
    uint32_t phase = 0;
    int t = 0;  // stage counter
    for (int it = 0; it < n_my; ++it) {
        const int g = (int)blockIdx.x + it * (int)gridDim.x;
        const int sys = g * SYS + s;
        const bool valid = sys < args.n_sys;

        // ------------------------------------------------------ forward pass
        double al[M], ga[M], de[M];  // rows 1..M-1 used (register resident)
        double ab0 = 0, cb0 = 0, db0 = 0;  // row 0 scaled by 1/b0
        double pi = 1.0, sa = 0.0, sd = 0.0;
#pragma unroll
        for (int k = 0; k < M; ++k) {
            if (ok) ok = mbar_wait_bounded(&full[slot], phase, args.status);
            const double* st = ring + (size_t)slot * 4 * T + tid;
            const double a = st[0], b = st[T], c = st[2 * T], d = st[3 * T];
            // The last warp to finish reading the slot refills it with stage
            // t + TILE_NST: the ring stays TILE_NST rows ahead of the slowest warp.
            __syncwarp();
            if ((tid & 31) == 0) {
                __threadfence_block();
                if (atomicAdd(&readers[slot], 1) == nwarps - 1) {
                    readers[slot] = 0;
                    if (ok && t + TILE_NST < total) issue(t + TILE_NST);
                }
            }
            ++t;
            if (++slot == TILE_NST) {
                slot = 0;
                phase ^= 1u;
            }
            if (k == 0) {
                const double ib = rcp_nr(b);
                ab0 = a * ib;
                cb0 = c * ib;
                db0 = d * ib;
            } else if (k == 1) {
                const double ib = rcp_nr(b);
                al[1] = a * ib;
                ga[1] = c * ib;
                de[1] = d * ib;
                sa = al[1];
                sd = de[1];
            } else {
                const double inv = rcp_nr(b - a * ga[k - 1]);
                ga[k] = c * inv;
                de[k] = (d - a * de[k - 1]) * inv;
                al[k] = -a * al[k - 1] * inv;
                if (k <= M - 2) {
                    pi = -ga[k - 1] * pi;
                    sa += pi * al[k];
                    sd += pi * de[k];
                }
            }
        }
        // reduced rows of this sub-segment
        const double pi_last = -ga[M - 2] * pi;  // pi_{M-1}
        const double r0 = rcp_nr(1.0 - cb0 * sa);
        const int i0 = 2 * q;
        {
            double* w = pb + i0 * SYS;
            w[0] = r0 * ab0;
            w[fs] = r0 * cb0 * pi_last;  // -r c0 gamma''_1, gamma''_1 = -pi_{M-1}
            w[2 * fs] = r0 * (db0 - cb0 * sd);
            w[SYS] = al[M - 1];
            w[fs + SYS] = ga[M - 1];
            w[2 * fs + SYS] = de[M - 1];
        }
        __syncthreads();

        // ------------------------------------------------- reduced system (PCR)
        // Row i: l_i x_{i-dl} + x_i + u_i x_{i+dl} = r_i.  Eliminating the rows
        // i-dl and i+dl doubles the coupling distance; out-of-range neighbours
        // are the zero guard rows (x = 0 there), or wrap around when periodic.
        int cur = 0;
        double x_first = 0.0, x_last = 0.0;
        bool solved = false;
        for (int dl = 1; dl < N; dl <<= 1) {
            const bool last_cyclic = CYCLIC && 2 * dl == N;
            const double* L = FB(cur, 0);
            const double* U = L + fs;
            const double* R = U + fs;
            double nl[2], nu[2], nr[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = i0 + h;
                int im = i - dl, ip = i + dl;
                if (CYCLIC) {
                    im = im < 0 ? im + N : im;
                    ip = ip >= N ? ip - N : ip;
                } else {
                    im = im < -1 ? -1 : im;
                    ip = ip > N ? N : ip;
                }
                const double li = L[i * SYS], ui = U[i * SYS], ri = R[i * SYS];
                const double lm = L[im * SYS], um = U[im * SYS], rm = R[im * SYS];
                const double lp = L[ip * SYS], up = U[ip * SYS], rp = R[ip * SYS];
                if (last_cyclic) {
                    // i-dl and i+dl are the same row j: 2x2 system in x_i, x_j
                    const double si = li + ui, sj = lm + um;
                    nr[h] = (ri - si * rm) * rcp_nr(1.0 - si * sj);
                    nl[h] = 0.0;
                    nu[h] = 0.0;
                } else {
                    const double ib = rcp_nr(1.0 - li * um - ui * lp);
                    nl[h] = -li * lm * ib;
                    nu[h] = -ui * up * ib;
                    nr[h] = (ri - li * rm - ui * rp) * ib;
                }
            }
            const int nxt = cur ^ 1;
            double* w = FB(nxt, 0) + i0 * SYS;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                w[h * SYS] = nl[h];
                w[fs + h * SYS] = nu[h];
                w[2 * fs + h * SYS] = nr[h];
            }
            if (last_cyclic) {
                x_first = nr[0];
                x_last = nr[1];
                solved = true;
            }
            __syncthreads();
            cur = nxt;
        }
        if (!solved) {
            const double* R = FB(cur, 2) + i0 * SYS;
            x_first = R[0];
            x_last = R[SYS];
        }

        // --------------------------------------------------- back substitution
        if (valid) {
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
        __syncthreads();  // PCR buffers are rewritten by the next group
    }
    if (!finite) raise_status(args.status, ST_NONFINITE);
    if (!ok && tid == 0) {
        // a wait gave up: give in-flight copies a bounded chance to land before
        // the CTA exits
        for (int i = 0; i < TILE_NST; ++i) mbar_wait_bounded(&full[i], 0, nullptr, 1u << 8);
    }
}

}  // namespace btdma
