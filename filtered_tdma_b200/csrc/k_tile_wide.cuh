// Wide-box variant of the register-tiled segmented solve (k_tile.cuh): twice the
// systems per CTA, so every row of a TMA box is twice as wide in HBM.
//
// Why: the DRAM serves a stream of row pieces (SYS x element bytes, rows a full
// row of the batch apart) at a rate that grows with the piece width: 64-byte
// pieces reach about half the bandwidth of 128-byte ones, 128-byte pieces about
// three quarters of 256-byte ones.  The tiled kernel keeps the elimination state
// of all its rows in registers, which caps it at 16 systems of 512 rows per SM
// (64-byte pieces for FP32 storage).  This kernel takes SYS = 512 / (NSEG / 2)
// systems (32 at 512 rows, 64 at 256) and holds only half of every group's state:
//
//   A0  sub-segments 0 .. H-1 (H = NSEG / 2), thread (s, q) = system s,
//       sub-segment q: the forward pass of k_tile.cuh reduced to its running
//       scalars; only the two reduced rows are kept.
//   A1  sub-segments H .. NSEG-1, thread (s, q) takes H + q: the same pass with
//       the per-row state in registers, as in k_tile.cuh.
//   reduced system: one warp-shuffle solve per system (reduced_solve_shfl).
//   B1  back substitution of A1's sub-segments from registers.
//   B0  the rows of A0 are loaded again (read earlier in the same group, mostly
//       still in L2), the forward pass is repeated with its state in registers,
//       and the back substitution follows.
//
// The ring (as in k_tile.cuh: full/empty mbarriers per stage, refills issued by
// a rotating producer warp; here with unhinted polls) carries 3 * SPG stages
// per group: A0, A1, B0.  B0's reads come mostly from L2: DRAM traffic measured
// 1.04x (FP32 storage) and 1.15x (FP64) the algorithmic 24 / 40 B/row at
// 262144 x 512.
// Every recurrence is the expression of k_tile.cuh; the two kernels agree to
// rounding (bit for bit where the compiler contracts the same multiply-adds).
// Needs NSEG = n_row / 16 even, 8 <= NSEG <= 32 (periodic: a power of two),
// n_sys * elem a multiple of 16 bytes and 16-byte aligned arrays; SYS = 32, 64
// or 128 for H in (8, 16], (4, 8] or [4, 4].
#pragma once

#include "btdma_common.cuh"
#include "k_reduced.cuh"
#include "k_tile.cuh"

namespace btdma {

// Shared memory: ring (NST stages x 4 arrays x RPS x T elements) + reduced rows
// (6 x NSEG x (SYS + 1) doubles; x_first / x_last reuse fields 0 and 1) +
// 2 NST mbarriers.
__host__ __device__ __forceinline__ size_t tile_wide_smem_bytes(int sys, int nseg, int nst,
                                                                int elem) {
    const size_t t = (size_t)sys * (nseg / 2);
    return (size_t)nst * 4 * tile_rps(elem) * t * elem + 6ull * nseg * (sys + 1) * sizeof(double) +
           2ull * nst * sizeof(uint64_t) + 128;
}

// Running state of one sub-segment's forward pass (rows 0 .. M-1).
struct WideFwd {
    double ab0, cb0, db0;  // row 0 scaled by its pivot
    double pi, sa, sd;     // running products of the reduced first row
    double alp, gap, dep;  // alpha, gamma, delta of the previous row
    double gm2;            // gamma of row M-2
};

// Row k of the forward pass (the expressions of k_tile.cuh's loop, FP64).
// KEEP: store alpha, gamma, delta of the row in al / ga / de.
template <bool KEEP>
__device__ __forceinline__ void wide_row(WideFwd& f, int k, double a, double b, double cc,
                                         double d, double* al, double* ga, double* de) {
    constexpr int M = TILE_MT;
    if (k == 0) {
        const double ib = rcp_nr(b);
        f.ab0 = a * ib;
        f.cb0 = cc * ib;
        f.db0 = d * ib;
    } else if (k == 1) {
        const double ib = rcp_nr(b);
        f.alp = a * ib;
        f.gap = cc * ib;
        f.dep = d * ib;
        f.pi = 1.0;
        f.sa = f.alp;
        f.sd = f.dep;
    } else {
        const double inv = rcp_nr(b - a * f.gap);
        const double g = cc * inv;
        const double e = (d - a * f.dep) * inv;
        const double l = -a * f.alp * inv;
        if (k <= M - 2) {
            f.pi = -f.gap * f.pi;
            f.sa += f.pi * l;
            f.sd += f.pi * e;
        }
        if (k == M - 2) f.gm2 = g;
        f.alp = l;
        f.gap = g;
        f.dep = e;
    }
    if constexpr (KEEP) {
        if (k >= 1) {
            al[k] = f.alp;
            ga[k] = f.gap;
            de[k] = f.dep;
        }
    }
}

// The two reduced rows of a finished sub-segment into red[f][q][s].
__device__ __forceinline__ void wide_reduced(const WideFwd& f, double* w, int fstride) {
    const double pi_last = -f.gm2 * f.pi;
    const double r0 = rcp_nr(1.0 - f.cb0 * f.sa);
    w[0 * fstride] = r0 * f.ab0;
    w[1 * fstride] = r0 * f.cb0 * pi_last;
    w[2 * fstride] = r0 * (f.db0 - f.cb0 * f.sd);
    w[3 * fstride] = f.alp;
    w[4 * fstride] = f.gap;
    w[5 * fstride] = f.dep;
}

// FILT: Filtered's reduced system (as tile_f64_kernel's FILT).
template <int SYS, bool CYCLIC, typename TIN, bool FILT = false>
__global__ void __launch_bounds__(TILE_MAX_THREADS, 1)
tile_wide_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmD,
                 const TileArgs args) {
    constexpr int M = TILE_MT;
    constexpr int RPS = tile_rps((int)sizeof(TIN));
    constexpr int SPG = M / RPS;    // stages per half sweep
    constexpr int SPT = 3 * SPG;    // stages per group: A0, A1, B0
    constexpr int RP = SYS + 1;
    extern __shared__ unsigned char smem_raw[];
    const int nseg = args.nseg, nst = args.nst;
    const int H = nseg / 2;
    const int T = SYS * H;  // == blockDim.x
    const int W = tile_lanes(nseg);
    const int fstride = nseg * RP;

    TIN* ring = reinterpret_cast<TIN*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const int sstride = 4 * RPS * T;  // elements per stage
    double* red = reinterpret_cast<double*>(ring + (size_t)nst * sstride);
    uint64_t* full = reinterpret_cast<uint64_t*>(red + 6 * fstride);
    uint64_t* empty = full + nst;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int nwarps = (T + 31) / 32;
    const int s = tid % SYS;
    const int ql = tid / SYS;
    const size_t ns = (size_t)args.n_sys;

    if (tid == 0) {
        for (int i = 0; i < nst; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], nwarps);
        }
        fence_mbar_init();
    }
    __syncthreads();

    // a closed gate leaves the CTA without groups (TILE_MODE_GATE_ZERO: the
    // gate is open while *gate == 0)
    const bool gated_off = args.gate != nullptr &&
                           ((*static_cast<const volatile unsigned*>(args.gate) == 0u) !=
                            ((args.mode & TILE_MODE_GATE_ZERO) != 0));
    const int filt_r = FILT ? (args.mode >> TILE_MODE_FILT_SHIFT) & 255 : 0;  // lanes a segment
    const int n_my = (!gated_off && args.n_groups > (int)blockIdx.x)
                         ? (args.n_groups - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x
                         : 0;
    const int total = n_my * SPT;
    const uint32_t stage_bytes = (uint32_t)sstride * sizeof(TIN);

    auto issue = [&](int t) {  // one thread
        const int slot = t % nst;
        const int g = (int)blockIdx.x + (t / SPT) * (int)gridDim.x;
        const int u = t % SPT;
        const int k0 = (u % SPG) * RPS;
        const int z = (u / SPG) == 1 ? H : 0;
        TIN* dst = ring + (size_t)slot * sstride;
        mbar_expect_tx(&full[slot], stage_bytes);
        tma_load_3d(dst + 0 * RPS * T, &tmA, g * SYS, k0, z, &full[slot]);
        tma_load_3d(dst + 1 * RPS * T, &tmB, g * SYS, k0, z, &full[slot]);
        tma_load_3d(dst + 2 * RPS * T, &tmC, g * SYS, k0, z, &full[slot]);
        tma_load_3d(dst + 3 * RPS * T, &tmD, g * SYS, k0, z, &full[slot]);
    };
    bool ok = true;
    if (tid == 0)
        for (int t = 0; t < nst && t < total; ++t) issue(t);

    const int toff = ql * RPS * SYS + s;
    const TIN* st = ring + toff;
    int slot = 0;
    uint32_t phase = 0;
    int pslot = nst - 1;
    uint32_t pphase = 1;
    int t = 0;
    int tw = 0;
    // Next stage's RPS rows of this thread's sub-segment (widened), then the
    // release of the slot and, one stage later, its refill.
    auto fetch = [&](double (&a2)[RPS], double (&b2)[RPS], double (&c2)[RPS], double (&d2)[RPS]) {
        if (ok) ok = mbar_wait_bounded_spin(&full[slot], phase, args.status);
#pragma unroll
        for (int r = 0; r < RPS; ++r) {
            a2[r] = (double)st[0 * RPS * T + r * SYS];
            b2[r] = (double)st[1 * RPS * T + r * SYS];
            c2[r] = (double)st[2 * RPS * T + r * SYS];
            d2[r] = (double)st[3 * RPS * T + r * SYS];
        }
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&empty[slot]);
            if (t >= 1 && warp == tw && t - 1 + nst < total && ok) {
                ok = mbar_wait_bounded_spin(&empty[pslot], pphase, args.status);
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
    };

    double nonfinite = 0.0;
    for (int it = 0; it < n_my; ++it) {
        const int g = (int)blockIdx.x + it * (int)gridDim.x;
        const int sys = g * SYS + s;
        const bool valid = sys < args.n_sys;
        const int q0 = ql, q1 = H + ql;

        // ------------------------------------------------ A0: scalars only
        {
            WideFwd f = {};
#pragma unroll
            for (int j = 0; j < SPG; ++j) {
                double a2[RPS], b2[RPS], c2[RPS], d2[RPS];
                fetch(a2, b2, c2, d2);
#pragma unroll
                for (int r = 0; r < RPS; ++r)
                    wide_row<false>(f, j * RPS + r, a2[r], b2[r], c2[r], d2[r], nullptr, nullptr,
                                    nullptr);
            }
            wide_reduced(f, red + q0 * RP + s, fstride);
        }
        // ------------------------------------------------ A1: state kept
        double al[M], ga[M], de[M];
        {
            WideFwd f = {};
#pragma unroll
            for (int j = 0; j < SPG; ++j) {
                double a2[RPS], b2[RPS], c2[RPS], d2[RPS];
                fetch(a2, b2, c2, d2);
#pragma unroll
                for (int r = 0; r < RPS; ++r)
                    wide_row<true>(f, j * RPS + r, a2[r], b2[r], c2[r], d2[r], al, ga, de);
            }
            wide_reduced(f, red + q1 * RP + s, fstride);
        }
        __syncthreads();

        // ------------------------------------------------ reduced system
        {
            const int per_pass = T / W;  // systems per pass
            const int p = tid % W;
            for (int base = 0; base < SYS; base += per_pass) {
                const int sp = base + tid / W;
                const bool act = sp < SYS && p < nseg;
                double l0 = 0, u0 = 0, r0 = 0, l1 = 0, u1 = 0, r1 = 0;
                double* src = red + p * RP + sp;
                if (act) {
                    l0 = src[0 * fstride];
                    u0 = src[1 * fstride];
                    r0 = src[2 * fstride];
                    l1 = src[3 * fstride];
                    u1 = src[4 * fstride];
                    r1 = src[5 * fstride];
                }
                double xf, xl;
                if constexpr (FILT)
                    reduced_solve_filtered<CYCLIC>(l0, u0, r0, l1, u1, r1, p, nseg, W, filt_r,
                                                   act, xf, xl);
                else
                    reduced_solve_shfl<CYCLIC>(l0, u0, r0, l1, u1, r1, p, nseg, W, act, xf, xl);
                if (act) {  // over the fields this thread has read
                    src[0] = xf;
                    src[fstride] = xl;
                }
            }
        }
        __syncthreads();

        // ------------------------------------------------ B1, B0
        auto back = [&](int q) {
            const double x_first = red[q * RP + s];
            const double x_last = red[fstride + q * RP + s];
            if (!valid) return;
            double* xp = args.X + (size_t)(q * M + M - 1) * ns + sys;
            *xp = x_last;
            double xn = x_last;
#pragma unroll
            for (int k = M - 2; k >= 1; --k) {
                xp -= ns;
                xn = de[k] - al[k] * x_first - ga[k] * xn;
                nonfinite = fma(xn, 0.0, nonfinite);
                *xp = xn;
            }
            xp -= ns;
            *xp = x_first;
            nonfinite = fma(x_first, 0.0, fma(x_last, 0.0, nonfinite));
        };
        back(q1);
        {
            WideFwd f = {};
#pragma unroll
            for (int j = 0; j < SPG; ++j) {
                double a2[RPS], b2[RPS], c2[RPS], d2[RPS];
                fetch(a2, b2, c2, d2);
#pragma unroll
                for (int r = 0; r < RPS; ++r)
                    wide_row<true>(f, j * RPS + r, a2[r], b2[r], c2[r], d2[r], al, ga, de);
            }
        }
        back(q0);
    }
    if (nonfinite != 0.0) raise_status(args.status, ST_NONFINITE);
    if (!ok && tid == 0)
        for (int i = 0; i < nst; ++i) mbar_wait_bounded(&full[i], 0, nullptr, 1u << 8);
}

}  // namespace btdma
