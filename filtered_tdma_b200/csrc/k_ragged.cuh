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
// The host sorts the systems into buckets of similar length and periodicity
// (so the shuffles of a warp are uniform), picks P per bucket (autotuner), and
// lays the work out as a task table: one entry per warp (this kernel) or per
// CTA (ragged_cta_kernel), so all buckets of one kind run in one launch.
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
    const int* list;       // system ids, bucket by bucket
    // Task table.  ragged_kernel: one entry per warp, {first list index, systems
    // (<= 32 / P), P, cyclic}; ragged_cta_kernel: one per CTA, {list index,
    // cyclic, 0, 0} (P = blockDim.x).
    const int4* tasks;
    int n_tasks;
    int mcap;              // ragged_kernel: state slots per lane (>= every task's rows per lane)
    unsigned* status;
    // ragged_persist_kernel: task counters per class (zero at launch), and each
    // class's first task and task count in the table
    int* next;
    int cls_first[3], cls_count[3];
    // ... and its warp class (counter next[3]): warp tasks of at most RAG_MT
    // rows a lane, table entries warp_first .. warp_first + warp_count - 1
    int warp_first, warp_count;
    // ragged_cta_kernel: CTA b prefetches the system of task b + pf_ahead (the
    // launch's co-resident CTAs: the task that takes over its slot) into L2;
    // 0: no prefetch
    int pf_ahead;
};

// Bulk prefetch into L2 of the 16-byte-aligned interior of elements
// [o, o + n) of one array (a hint: nothing waits for it and it cannot fault;
// the at most 15 bytes at either end outside the aligned interior are left out).
template <typename TIN>
__device__ __forceinline__ void rag_prefetch_l2(const void* arr, long long o, int n) {
    const size_t b = __cvta_generic_to_global(static_cast<const TIN*>(arr) + o);
    const size_t e = b + (size_t)n * sizeof(TIN);
    const size_t b16 = (b + 15) & ~(size_t)15, e16 = e & ~(size_t)15;
    if (e16 > b16)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b16),
                     "r"((unsigned)(e16 - b16))
                     : "memory");
}

// The four input arrays of system sys (one thread issues it).
template <typename TIN>
__device__ __forceinline__ void rag_prefetch_system(const RagArgs& a, int sys) {
    const long long o = a.off[sys];
    const int n = (int)(a.off[sys + 1] - o);
    rag_prefetch_l2<TIN>(a.A, o, n);
    rag_prefetch_l2<TIN>(a.B, o, n);
    rag_prefetch_l2<TIN>(a.C, o, n);
    rag_prefetch_l2<TIN>(a.D, o, n);
}

constexpr int RAG_LOOKAHEAD = 4;  // rows loaded ahead of the elimination

// Shared memory per warp: 3 fields x mcap rows x 32 lanes doubles.
__host__ __device__ constexpr size_t rag_smem_bytes(int warps, int mcap) {
    return (size_t)warps * 3 * mcap * 32 * sizeof(double);
}

// One warp task {first list index, systems (<= 32 / P), P, cyclic}, solved by
// the calling warp (this thread: lane); its state area of 3 x mcap x 32
// doubles starts at wsm.
template <typename TIN>
__device__ __forceinline__ void rag_warp_body(const RagArgs& a, const int4 task, double* wsm,
                                              const int lane, const int mcap) {
    const int P = task.z;
    const int g = lane / P;
    const int p = lane % P;
    const bool cyclic = task.w != 0;  // uniform over the warp
    double* st = wsm + lane;  // field f, row k: st[(f*mcap+k)*32]

    const bool have = g < task.y;
    int m = 0;
    long long row0 = 0;
    if (have) {
        const int sys = a.list[task.x + g];
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
        // rows k0 .. k0 + RAG_LOOKAHEAD - 1, clamped (in bounds) at the tail; the
        // next batch is requested before the current one is eliminated
        double ra[RAG_LOOKAHEAD], rb[RAG_LOOKAHEAD], rc[RAG_LOOKAHEAD], rd[RAG_LOOKAHEAD];
        auto fetch = [&](int k0, double* fa, double* fb, double* fc, double* fd) {
#pragma unroll
            for (int j = 0; j < RAG_LOOKAHEAD; ++j) {
                const int k = k0 + j < m ? k0 + j : m - 1;
                fa[j] = (double)__ldg(pA + k);
                fb[j] = (double)__ldg(pB + k);
                fc[j] = (double)__ldg(pC + k);
                fd[j] = (double)__ldg(pD + k);
            }
        };
        fetch(0, ra, rb, rc, rd);
        for (int k0 = 0; k0 < m; k0 += RAG_LOOKAHEAD) {
            double na[RAG_LOOKAHEAD], nb[RAG_LOOKAHEAD], nc[RAG_LOOKAHEAD], nd[RAG_LOOKAHEAD];
            fetch(k0 + RAG_LOOKAHEAD, na, nb, nc, nd);
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
#pragma unroll
            for (int j = 0; j < RAG_LOOKAHEAD; ++j) {
                ra[j] = na[j];
                rb[j] = nb[j];
                rc[j] = nc[j];
                rd[j] = nd[j];
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
    if (cyclic)
        reduced_solve_shfl<true>(l0, u0, r0, l1, u1, r1, p, P, P, act, xf, xl);
    else
        reduced_solve_shfl<false>(l0, u0, r0, l1, u1, r1, p, P, P, act, xf, xl);

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

template <typename TIN>
__global__ void __launch_bounds__(256) ragged_kernel(const RagArgs a) {
    extern __shared__ double rsm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * (blockDim.x >> 5) + warp;
    if (gw >= a.n_tasks) return;  // the whole warp
    rag_warp_body<TIN>(a, a.tasks[gw], rsm + (size_t)warp * 3 * a.mcap * 32, lane, a.mcap);
}

// Long systems: one CTA of P threads (P a power of two, 64..512) per system,
// at most RAG_MT rows per thread, the elimination state in shared memory laid
// out [field][row][thread] (consecutive threads, consecutive doubles).  The
// reduced system of the P sub-segments goes through shared memory: one
// cyclic-reduction level leaves P unknowns, which warp 0 solves in two levels
// (groups of P / 32 rows, then the 32 groups' interfaces with
// reduced_solve_shfl; see rag_cta_body).
constexpr int RAG_MT = 16;

// STAGED: A, C and D of the whole system are first copied into shared memory
// with coalesced loads (B, read by the forward sweep only, goes to registers:
// each thread requests its rows before the fill, so one memory latency covers
// both), laid out [array][thread][row of segment]
// with RAG_MT slots per thread and the row index XOR-swizzled by the thread's
// low four bits (slot k ^ (p & 15)): consecutive rows of a segment land in
// distinct banks for the coalesced fill, and the threads reading row k of
// their segments hit distinct banks too, with no padding.  The elimination
// state then overwrites A, C, D in place, x overwrites D during the back
// substitution and leaves with coalesced stores.  At 4096 rows (256 threads of
// 16 rows) a staged CTA takes 110 KB, so two fit on an SM and one's fill
// overlaps the other's sweeps.  Without staging each thread reads its
// contiguous rows straight from global memory, which leaves L1 to hold four
// lines per thread.
// mcap: rows per thread of the launch (<= RAG_MT).
__host__ __device__ __forceinline__ int rag_slot(int p, int k) { return k ^ (p & 15); }
// Shared memory of one system: the sub-segments' first rows (3 fields of P + 2
// with zero guards), the interface system in the group layout (3 fields of 33
// slots per row of a group, see rag_cta_body) and the state / staging area.
__host__ __device__ constexpr size_t rag_cta_smem_bytes(int P, bool staged, int mcap) {
    return (3ull * (P + 2) + 3ull * 33 * (size_t)(P / 32) +
            (staged ? 3ull * RAG_MT * P : 3ull * (size_t)mcap * P)) *
           sizeof(double);
}

// Asynchronous global -> shared copy of one element (completion:
// cp.async.wait_all) into the 8-byte slot dst: a double fills it, a float its
// low word.
__device__ __forceinline__ void cp_async_elem(double* dst, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_elem(double* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}

// r / d = __umulhi(r, rag_magic(d)) exactly for d >= 2 and r * d < 2^32:
// rag_magic(d) = ceil(2^32 / d) = 2^32 / d + e / d with 0 <= e < d, so the
// product's high word is floor(r / d + r e / (d 2^32)), and r e / 2^32 < 1
// cannot carry the fraction (r mod d) / d <= (d - 1) / d past the next integer.
__device__ __forceinline__ unsigned rag_magic(int d) { return 0xFFFFFFFFu / (unsigned)d + 1u; }

// (segment, row in segment) of row r of a system split by para_range into P
// parts of base or base + 1 rows (the first rem parts longer, split = rem *
// (base + 1) rows in all); mag0 / mag1 = rag_magic(base) / rag_magic(base + 1).
// Rows per system stay below 2^13 and base + 1 below 2^5.
__device__ __forceinline__ void rag_locate(int r, int base, int rem, int split, unsigned mag0,
                                           unsigned mag1, int& q, int& k) {
    const bool lo = r < split;
    const int rr = lo ? r : r - split;
    const int qq = (int)__umulhi((unsigned)rr, lo ? mag1 : mag0);
    k = rr - qq * (lo ? base + 1 : base);
    q = lo ? qq : qq + rem;
}

// One system (task {list index, cyclic, ...}) solved by a group of P threads
// (thread p of the group), whose barrier is bar.sync bid, P (bid 0 with the
// whole CTA: __syncthreads) and whose shared memory starts at rsm.
template <typename TIN, bool STAGED>
__device__ __forceinline__ void rag_cta_body(const RagArgs& a, const int4 task, const int P,
                                             double* rsm, const int p, const int bid) {
    constexpr int M = RAG_MT;
    const int NT = P;
    const bool act = p < P;
    auto gsync = [&]() { asm volatile("bar.sync %0, %1;" ::"r"(bid), "r"(P) : "memory"); };
    const int gs = P + 2;  // guard rows at 0 and P + 1 stay zero (non-periodic ends)
    // first rows of the sub-segments: field f of sub-segment row at F(f, row)
    auto F = [&](int f, int row) -> double& { return rsm[f * gs + row + 1]; };
    if (p < 3) {
        rsm[p * gs] = 0.0;
        rsm[p * gs + P + 1] = 0.0;
    }

    const bool cyclic = task.y != 0;  // uniform over the CTA
    const int sys = a.list[task.x];
    const long long o = a.off[sys];
    const int n = (int)(a.off[sys + 1] - o);
    const int base = n / P, rem = n % P;
    const int m = act ? base + (p < rem ? 1 : 0) : 0;  // 3 <= m <= M (host's choice of P)
    const long long row0 = o + (long long)p * base + (p < rem ? p : rem);
    const TIN* __restrict__ pA = static_cast<const TIN*>(a.A) + row0;
    const TIN* __restrict__ pB = static_cast<const TIN*>(a.B) + row0;
    const TIN* __restrict__ pC = static_cast<const TIN*>(a.C) + row0;
    const TIN* __restrict__ pD = static_cast<const TIN*>(a.D) + row0;

    // interface system, group layout (below): row q, field f at T[f * TS + TI(q)]
    const int G = P >> 5, lg = __ffs(G) - 1, TS = 33 * G;
    double* const T = rsm + 3 * gs;
    auto TI = [&](int q) { return (q & (G - 1)) * 33 + (q >> lg); };
    double* const stg = T + 3 * TS;  // state / staging area
    // this thread's slots (mcap = the launch's rows per thread, <= M):
    // unstaged [field][row][thread] -> stt[(f * mcap + k) * P];
    // staged [field][thread][slot] -> stt[f * P * M + rag_slot(p, k)]
    double* stt = STAGED ? stg + p * M : stg + p;
    const int fs = STAGED ? P * M : a.mcap * P;  // field stride
    const int ks = STAGED ? 1 : P;               // row stride (unstaged)
    // rows per thread: base or base + 1; mx, the most, is the same for the
    // whole group (the B loads stop there)
    const int mx = base + (rem > 0 ? 1 : 0);
    const int split = rem * (base + 1);
    const unsigned mag0 = rag_magic(base > 1 ? base : 2), mag1 = rag_magic(base + 1);
    // staged: the thread's B rows go to registers, requested before the fill so
    // that both arrive together and the forward sweep waits on shared memory only
    // (rows past m repeat row m - 1 and are never used)
    double bq[M];
    if constexpr (STAGED) {
#pragma unroll
        for (int k = 0; k < M; ++k) {
            double v = 0.0;
            if (k < mx) v = (double)__ldg(pB + (k < m ? k : m - 1));
            bq[k] = v;
        }
    }
    if constexpr (STAGED) {
        // fields 0..2 = A, C, D; coalesced over the system's rows
        const TIN* __restrict__ gA = static_cast<const TIN*>(a.A) + o;
        const TIN* __restrict__ gC = static_cast<const TIN*>(a.C) + o;
        const TIN* __restrict__ gD = static_cast<const TIN*>(a.D) + o;
        // asynchronous copies straight into the staged layout, every row of the
        // thread in flight at once; FP32 values land in the low word of their
        // 8-byte slot and each thread widens its own rows once they are in
        for (int r = p; r < n; r += NT) {
            int q, k;
            rag_locate(r, base, rem, split, mag0, mag1, q, k);
            double* dst = stg + q * M + rag_slot(q, k);
            cp_async_elem(dst + 0 * fs, gA + r);
            cp_async_elem(dst + 1 * fs, gC + r);
            cp_async_elem(dst + 2 * fs, gD + r);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        gsync();
        if constexpr (sizeof(TIN) == 4) {
            for (int k = 0; k < m; ++k)
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                    double* sl = stt + f * fs + rag_slot(p, k);
                    *sl = (double)*reinterpret_cast<const float*>(sl);
                }
        }
    }
    // slot of row k: staged swizzled, unstaged [row][thread]
    auto SL = [&](int k) { return STAGED ? rag_slot(p, k) : k * ks; };
    // state: alpha, gamma, delta (in place of A, C, D when staged)
    auto AL = [&](int k) -> double& { return stt[0 * fs + SL(k)]; };
    auto GA = [&](int k) -> double& { return stt[1 * fs + SL(k)]; };
    auto DE = [&](int k) -> double& { return stt[2 * fs + SL(k)]; };
    double ab0 = 0, cb0 = 0, db0 = 0, pi = 1.0, sa = 0.0, sd = 0.0, pi_last = 0.0;
    double alp = 0, gap = 0, dep = 0;  // row k-1
    if (act) {
    // rows of batch k0 .. k0 + RAG_LOOKAHEAD - 1 (clamped in bounds); the next
    // batch is requested before the current one is eliminated
    double ra[RAG_LOOKAHEAD], rb[RAG_LOOKAHEAD], rc[RAG_LOOKAHEAD], rd[RAG_LOOKAHEAD];
    auto fetch = [&](int k0, double* fa, double* fb, double* fc, double* fd) {
#pragma unroll
        for (int j = 0; j < RAG_LOOKAHEAD; ++j) {
            const int kk = k0 + j < m ? k0 + j : m - 1;
            if constexpr (STAGED) {
                const int sl = rag_slot(p, kk);
                fa[j] = stt[0 * fs + sl];
                fb[j] = bq[k0 + j];  // k0 + j < M: a register
                fc[j] = stt[1 * fs + sl];
                fd[j] = stt[2 * fs + sl];
            } else {
                fa[j] = (double)__ldg(pA + kk);
                fb[j] = (double)__ldg(pB + kk);
                fc[j] = (double)__ldg(pC + kk);
                fd[j] = (double)__ldg(pD + kk);
            }
        }
    };
    fetch(0, ra, rb, rc, rd);
#pragma unroll
    for (int k0 = 0; k0 < M; k0 += RAG_LOOKAHEAD) {
        double na[RAG_LOOKAHEAD], nb[RAG_LOOKAHEAD], nc[RAG_LOOKAHEAD], nd[RAG_LOOKAHEAD];
        if (k0 + RAG_LOOKAHEAD < M) fetch(k0 + RAG_LOOKAHEAD, na, nb, nc, nd);
#pragma unroll
        for (int j = 0; j < RAG_LOOKAHEAD; ++j) {
            const int k = k0 + j;
            if (k >= m) continue;
            if (k == 0) {
                const double ib = rcp_nr(rb[j]);
                ab0 = ra[j] * ib;
                cb0 = rc[j] * ib;
                db0 = rd[j] * ib;
            } else {
                double al, ga, de;
                if (k == 1) {
                    const double ib = rcp_nr(rb[j]);
                    al = ra[j] * ib;
                    ga = rc[j] * ib;
                    de = rd[j] * ib;
                    sa = al;
                    sd = de;
                } else {
                    const double inv = rcp_nr(rb[j] - ra[j] * gap);
                    ga = rc[j] * inv;
                    de = (rd[j] - ra[j] * dep) * inv;
                    al = -ra[j] * alp * inv;
                    if (k <= m - 2) {
                        pi = -gap * pi;
                        sa += pi * al;
                        sd += pi * de;
                    }
                    if (k == m - 1) pi_last = -gap * pi;
                }
                AL(k) = al;
                GA(k) = ga;
                DE(k) = de;
                alp = al;
                gap = ga;
                dep = de;
            }
        }
        if (k0 + RAG_LOOKAHEAD < M) {
#pragma unroll
            for (int j = 0; j < RAG_LOOKAHEAD; ++j) {
                ra[j] = na[j];
                rb[j] = nb[j];
                rc[j] = nc[j];
                rd[j] = nd[j];
            }
        }
    }
    }  // act
    const double l1 = alp, u1 = gap, r1 = dep;  // row m - 1
    const double rr = rcp_nr(1.0 - cb0 * sa);
    const double l0 = rr * ab0, u0 = rr * cb0 * pi_last, r0 = rr * (db0 - cb0 * sd);

    // ---------------------------------------------- reduced system (shared memory)
    // One cyclic-reduction level leaves the interface system in the last-row
    // unknowns (unit diagonal, as in reduced_solve_shfl):
    //   a_q xL(q-1) + xL(q) + c_q xL(q+1) = d_q,  q = 0 .. P-1.
    // Warp 0 of the group solves it in two levels: lane t takes the G = P / 32
    // consecutive rows t G .. t G + G - 1 and runs the modified Thomas steps of
    // the sweep above on them (unit diagonal), the 32 groups' own interface
    // rows go through reduced_solve_shfl, and each lane back-substitutes its
    // group.  Group layout: row q at slot (q % G) * 33 + q / G of each field,
    // so lane t's k-th row sits at k * 33 + t (the warp reads consecutive
    // slots) and the other threads' writes and reads of row p land in distinct
    // banks up to 2-way.  Three barriers per system.
    if (act) {
        F(0, p) = l0;
        F(1, p) = u0;
        F(2, p) = r0;
    }
    gsync();
    if (act) {
        const int pn = (cyclic && p == P - 1) ? 0 : p + 1;  // p + 1 == P: the zero guard
        const double l0n = F(0, pn), u0n = F(1, pn), r0n = F(2, pn);
        const double ib = rcp_nr(1.0 - l1 * u0 - u1 * l0n);
        const int ti = TI(p);
        T[ti] = -l1 * l0 * ib;
        T[TS + ti] = -u1 * u0n * ib;
        T[2 * TS + ti] = (r1 - l1 * r0 - u1 * r0n) * ib;
    }
    gsync();
    if (p < 32) {  // warp 0 of the group (P >= 64: whole warps)
        double* const ta = T + p;
        double* const tc = T + TS + p;
        double* const td = T + 2 * TS + p;
        double gl0, gu0, gr0, gl1, gu1, gr1;  // the group's interface rows
        if (G == 2) {  // no interior: the two rows are the interface rows
            gl0 = ta[0], gu0 = tc[0], gr0 = td[0];
            gl1 = ta[33], gu1 = tc[33], gr1 = td[33];
        } else {
            const double ab0 = ta[0], cb0 = tc[0], db0 = td[0];
            // row 1 with unit diagonal: alpha, gamma, delta are its a, c, d
            double alp = ta[33], gap = tc[33], dep = td[33];
            double gpi = 1.0, gsa = alp, gsd = dep, gpi_last = 0.0;
            for (int k = 2; k < G; ++k) {
                const double av = ta[k * 33], cv = tc[k * 33], dv = td[k * 33];
                const double inv = rcp_nr(1.0 - av * gap);
                const double ga = cv * inv, de = (dv - av * dep) * inv, al = -av * alp * inv;
                if (k <= G - 2) {
                    gpi = -gap * gpi;
                    gsa += gpi * al;
                    gsd += gpi * de;
                } else {
                    gpi_last = -gap * gpi;
                }
                ta[k * 33] = al;
                tc[k * 33] = ga;
                td[k * 33] = de;
                alp = al;
                gap = ga;
                dep = de;
            }
            const double rr = rcp_nr(1.0 - cb0 * gsa);
            gl0 = rr * ab0, gu0 = rr * cb0 * gpi_last, gr0 = rr * (db0 - cb0 * gsd);
            gl1 = alp, gu1 = gap, gr1 = dep;
        }
        double gxf, gxl;
        if (cyclic)
            reduced_solve_shfl<true>(gl0, gu0, gr0, gl1, gu1, gr1, p, 32, 32, true, gxf, gxl);
        else
            reduced_solve_shfl<false>(gl0, gu0, gr0, gl1, gu1, gr1, p, 32, 32, true, gxf, gxl);
        // x of the group's rows overwrite their delta
        td[(G - 1) * 33] = gxl;
        double gxn = gxl;
        for (int k = G - 2; k >= 1; --k) {
            gxn = td[k * 33] - ta[k * 33] * gxf - tc[k * 33] * gxn;
            td[k * 33] = gxn;
        }
        td[0] = gxf;
    }
    gsync();
    double xl = 0.0, xlm = 0.0;
    if (act) {
        xl = T[2 * TS + TI(p)];
        if (cyclic)
            xlm = T[2 * TS + TI(p == 0 ? P - 1 : p - 1)];
        else
            xlm = p == 0 ? 0.0 : T[2 * TS + TI(p - 1)];
    }
    const double xf = act ? r0 - l0 * xlm - u0 * xl : 0.0;

    // ------------------------------------------------ back substitution
    double* xp = a.X + row0;
    double nonfinite = fma(xf, 0.0, fma(xl, 0.0, 0.0));
    double xn = xl;
    // staged: x overwrites delta in the D field (each row's delta is read just
    // before) and leaves coalesced
    auto XO = [&](int k) -> double& { return stt[2 * fs + SL(k)]; };
#pragma unroll 4
    for (int k = m - 2; k >= 1; --k) {
        {
            xn = DE(k) - AL(k) * xf - GA(k) * xn;
            nonfinite = fma(xn, 0.0, nonfinite);
            if constexpr (STAGED)
                XO(k) = xn;
            else
                xp[k] = xn;
        }
    }
    if constexpr (STAGED) {
        if (act) {
            XO(0) = xf;
            XO(m - 1) = xl;
        }
        gsync();
        double* gX = a.X + o;
        for (int r = p; r < n; r += NT) {
            int q, k;
            rag_locate(r, base, rem, split, mag0, mag1, q, k);
            gX[r] = stg[2 * fs + q * M + rag_slot(q, k)];
        }
    } else if (act) {
        xp[0] = xf;
        xp[m - 1] = xl;
    }
    if (nonfinite != 0.0) raise_status(a.status, ST_NONFINITE);  // NaN != 0
}

// One launch per bucket shape: one system per CTA of P = blockDim.x threads.
template <typename TIN, bool STAGED>
__global__ void __launch_bounds__(512) ragged_cta_kernel(const RagArgs a) {
    extern __shared__ double rsm[];
    if (threadIdx.x == 0 && a.pf_ahead > 0 && (int)blockIdx.x + a.pf_ahead < a.n_tasks)
        rag_prefetch_system<TIN>(a, a.list[a.tasks[blockIdx.x + a.pf_ahead].x]);
    rag_cta_body<TIN, STAGED>(a, a.tasks[blockIdx.x], (int)blockDim.x, rsm, (int)threadIdx.x, 0);
}

// Persistent form: every long system of the plan in one launch.  CTAs of
// RAG_PERSIST_THREADS threads (two per SM) work through three classes of
// tasks {list index, cyclic, P, staged} (P = 256, 128, 64: the shape each
// bucket was tuned to), each class's tasks in the table's order (longest
// first) from its own counter a.next[c] (zeroed before the launch).  In class
// c the CTA splits into 2^c groups of P threads, each with its own named
// barrier and shared-memory slice, taking tasks independently; a group moves
// on to the next class when its class is drained (the next class's groups lie
// inside it, with barriers of their own).  A group claims its next task before
// solving the current one and prefetches that system into L2, so its fill
// reads L2 instead of waiting on DRAM.  Last, every warp takes warp tasks
// (short systems, P lanes each) from counter a.next[3] on its own, in half of
// its 64-thread group's slice, which that group has left (both its warps leave
// the last CTA class together), so the short work fills the launch's tail.
// a.mcap must be RAG_MT.
constexpr int RAG_PERSIST_THREADS = 256;
constexpr int RAG_PERSIST_CLASSES = 3;
// shared-memory slice of a group of P threads (nested: two slices of P / 2
// fit in one of P)
__host__ __device__ constexpr size_t rag_persist_slice(int P) {
    return rag_cta_smem_bytes(64, true, RAG_MT) * (size_t)(P / 64);
}
static_assert(rag_cta_smem_bytes(128, true, RAG_MT) <= rag_persist_slice(128) &&
                  rag_cta_smem_bytes(256, true, RAG_MT) <= rag_persist_slice(256),
              "a group's shared memory fits its slice");
static_assert(2 * rag_smem_bytes(1, RAG_MT) <= rag_persist_slice(64),
              "a 64-thread group's two warps' warp-task state fits its slice");
template <typename TIN>
__global__ void __launch_bounds__(RAG_PERSIST_THREADS, 2) ragged_persist_kernel(const RagArgs a) {
    extern __shared__ double rsm[];
    // claimed tasks by barrier id (unique per group), two slots: the one written
    // in an iteration is read after its barriers, and rewritten two iterations on
    __shared__ int next_task[2][1 << RAG_PERSIST_CLASSES];
    const int tid = threadIdx.x;
    static_assert(RAG_PERSIST_CLASSES == 3, "class selects below");
    for (int c = 0; c < RAG_PERSIST_CLASSES; ++c) {
        const int P = RAG_PERSIST_THREADS >> c;
        const int g = tid / P, p = tid % P;
        const int bid = (1 << c) + g;  // 1; 2, 3; 4 .. 7
        double* sm = rsm + rag_persist_slice(P) / sizeof(double) * g;
        // constant indices: an index computed at run time would copy the whole
        // parameter block to local memory
        const int ccount = c == 0 ? a.cls_count[0] : c == 1 ? a.cls_count[1] : a.cls_count[2];
        const int cfirst = c == 0 ? a.cls_first[0] : c == 1 ? a.cls_first[1] : a.cls_first[2];
        if (p == 0) next_task[0][bid] = atomicAdd(&a.next[c], 1);
        asm volatile("bar.sync %0, %1;" ::"r"(bid), "r"(P) : "memory");
        int t = next_task[0][bid];
        for (int it = 1; t < ccount; ++it) {
            const int4 task = a.tasks[cfirst + t];
            if (p == 0) {
                const int tn = atomicAdd(&a.next[c], 1);
                next_task[it & 1][bid] = tn;
                if (tn < ccount) rag_prefetch_system<TIN>(a, a.list[a.tasks[cfirst + tn].x]);
            }
            if (task.w)
                rag_cta_body<TIN, true>(a, task, P, sm, p, bid);
            else
                rag_cta_body<TIN, false>(a, task, P, sm, p, bid);
            // the group's shared memory is rewritten by its next task
            asm volatile("bar.sync %0, %1;" ::"r"(bid), "r"(P) : "memory");
            t = next_task[it & 1][bid];
        }
    }
    const int lane = tid & 31, warp = tid >> 5;
    double* wsm = rsm + rag_persist_slice(64) / sizeof(double) * (warp >> 1) +
                  (size_t)(warp & 1) * (rag_smem_bytes(1, RAG_MT) / sizeof(double));
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(&a.next[3], 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= a.warp_count) break;
        rag_warp_body<TIN>(a, a.tasks[a.warp_first + t], wsm, lane, RAG_MT);
        __syncwarp();  // the warp's state area is rewritten by its next task
    }
}

// Interleaved layout of one bucket (the autotuner's alternative to solving it
// in place): its `count` non-periodic systems, list[first .. first + count),
// copied into a row-interleaved batch of npad rows x nbp systems (row r of
// system j at r * nbp + j; npad a multiple of 16, nbp of 4), which the tiled
// kernel then solves like any uniform batch.  A system shorter than npad is
// continued by identity rows (a = c = d = 0, b = 1) and its own A[first] and
// C[last], which a non-periodic system does not use, are stored as zero, so the
// padding neither couples to it nor changes its solution; columns past count
// are identity systems.  32 x 32 tiles through shared memory: read along each
// system's contiguous rows, write along the interleaved rows.
constexpr int RAG_IL_TILE = 32;

template <typename TIN>
__global__ void __launch_bounds__(256) rag_gather_kernel(const TIN* __restrict__ A,
                                                          const TIN* __restrict__ B,
                                                          const TIN* __restrict__ C,
                                                          const TIN* __restrict__ D,
                                                          const long long* __restrict__ off,
                                                          const int* __restrict__ list, int first,
                                                          int count, int npad, int nbp,
                                                          TIN* __restrict__ out) {
    __shared__ TIN t[4][RAG_IL_TILE][RAG_IL_TILE + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    const int j0 = blockIdx.x * RAG_IL_TILE, r0 = blockIdx.y * RAG_IL_TILE;
    const size_t plane = (size_t)npad * nbp;
    for (int jj = ty; jj < RAG_IL_TILE; jj += 8) {
        const int j = j0 + jj, r = r0 + tx;
        TIN a = 0, b = 1, c = 0, d = 0;
        if (j < count) {
            const int sys = list[first + j];
            const long long o = off[sys];
            const int n = (int)(off[sys + 1] - o);
            if (r < n) {
                a = r == 0 ? TIN(0) : A[o + r];
                b = B[o + r];
                c = r == n - 1 ? TIN(0) : C[o + r];
                d = D[o + r];
            }
        }
        t[0][jj][tx] = a;
        t[1][jj][tx] = b;
        t[2][jj][tx] = c;
        t[3][jj][tx] = d;
    }
    __syncthreads();
    for (int rr = ty; rr < RAG_IL_TILE; rr += 8) {
        const int r = r0 + rr, j = j0 + tx;
        if (r < npad && j < nbp) {
            const size_t e = (size_t)r * nbp + j;
#pragma unroll
            for (int f = 0; f < 4; ++f) out[f * plane + e] = t[f][tx][rr];
        }
    }
}

// The solution back from the interleaved batch to the systems' rows.
__global__ void __launch_bounds__(256) rag_scatter_kernel(const double* __restrict__ xi,
                                                           const long long* __restrict__ off,
                                                           const int* __restrict__ list,
                                                           int first, int count, int npad,
                                                           int nbp, double* __restrict__ X) {
    __shared__ double t[RAG_IL_TILE][RAG_IL_TILE + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int j0 = blockIdx.x * RAG_IL_TILE, r0 = blockIdx.y * RAG_IL_TILE;
    for (int rr = ty; rr < RAG_IL_TILE; rr += 8) {
        const int r = r0 + rr, j = j0 + tx;
        t[rr][tx] = (r < npad && j < nbp) ? xi[(size_t)r * nbp + j] : 0.0;
    }
    __syncthreads();
    for (int jj = ty; jj < RAG_IL_TILE; jj += 8) {
        const int j = j0 + jj, r = r0 + tx;
        if (j < count) {
            const int sys = list[first + j];
            const long long o = off[sys];
            if (r < (int)(off[sys + 1] - o)) X[o + r] = t[tx][jj];
        }
    }
}

}  // namespace btdma
