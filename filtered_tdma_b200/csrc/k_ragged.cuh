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
};

constexpr int RAG_LOOKAHEAD = 4;  // rows loaded ahead of the elimination

// Shared memory per warp: 3 fields x mcap rows x 32 lanes doubles.
__host__ __device__ __forceinline__ size_t rag_smem_bytes(int warps, int mcap) {
    return (size_t)warps * 3 * mcap * 32 * sizeof(double);
}

template <typename TIN>
__global__ void __launch_bounds__(256) ragged_kernel(const RagArgs a) {
    extern __shared__ double rsm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * (blockDim.x >> 5) + warp;
    if (gw >= a.n_tasks) return;  // the whole warp
    const int4 task = a.tasks[gw];
    const int P = task.z;
    const int g = lane / P;
    const int p = lane % P;
    const bool cyclic = task.w != 0;  // uniform over the warp
    const int mcap = a.mcap;
    double* st = rsm + (size_t)warp * 3 * mcap * 32 + lane;  // field f, row k: st[(f*mcap+k)*32]

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

// Long systems: one CTA of P threads (P a power of two, 64..512) per system,
// at most RAG_MT rows per thread, the elimination state in shared memory laid
// out [field][row][thread] (consecutive threads, consecutive doubles).  The
// reduced system of the P sub-segments runs through shared memory: one
// cyclic-reduction level, then parallel cyclic reduction with a block barrier
// per level (the same steps as reduced_solve_shfl).
constexpr int RAG_MT = 16;

// STAGED: A, C and D of the whole system are first copied into shared memory
// with coalesced loads (B, read by the forward sweep only, comes straight from
// global memory a few rows ahead), laid out [array][thread][row of segment]
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
__host__ __device__ __forceinline__ size_t rag_cta_smem_bytes(int P, bool staged, int mcap) {
    return (2ull * 3 * (P + 2) +
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

// (segment, row in segment) of row r of a system split by para_range into P
// parts of base or base + 1 rows (the first rem parts longer).
__device__ __forceinline__ void rag_locate(int r, int base, int rem, float inv0, float inv1,
                                           int& q, int& k) {
    const int split = rem * (base + 1);
    if (r < split) {
        q = (int)((float)r * inv1);
        if (q * (base + 1) > r) --q;
        else if ((q + 1) * (base + 1) <= r) ++q;
        k = r - q * (base + 1);
    } else {
        const int r2 = r - split;
        q = (int)((float)r2 * inv0);
        if (q * base > r2) --q;
        else if ((q + 1) * base <= r2) ++q;
        k = r2 - q * base;
        q += rem;
    }
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
    auto F = [&](int b, int f, int row) -> double& { return rsm[(b * 3 + f) * gs + row + 1]; };
    if (p < 6) {
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

    double* const stg = rsm + 2 * 3 * gs;  // state / staging area
    // this thread's slots (mcap = the launch's rows per thread, <= M):
    // unstaged [field][row][thread] -> stt[(f * mcap + k) * P];
    // staged [field][thread][slot] -> stt[f * P * M + rag_slot(p, k)]
    double* stt = STAGED ? stg + p * M : stg + p;
    const int fs = STAGED ? P * M : a.mcap * P;  // field stride
    const int ks = STAGED ? 1 : P;               // row stride (unstaged)
    const float inv0 = 1.0f / (float)(base > 0 ? base : 1), inv1 = 1.0f / (float)(base + 1);
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
            rag_locate(r, base, rem, inv0, inv1, q, k);
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
                fb[j] = (double)__ldg(pB + kk);
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
    if (act) {
        F(1, 0, p) = l0;
        F(1, 1, p) = u0;
        F(1, 2, p) = r0;
    }
    gsync();
    if (act) {
        const int pn = (cyclic && p == P - 1) ? 0 : p + 1;  // p + 1 == P: the zero guard
        const double l0n = F(1, 0, pn), u0n = F(1, 1, pn), r0n = F(1, 2, pn);
        const double ib = rcp_nr(1.0 - l1 * u0 - u1 * l0n);
        F(0, 0, p) = -l1 * l0 * ib;
        F(0, 1, p) = -u1 * u0n * ib;
        F(0, 2, p) = (r1 - l1 * r0 - u1 * r0n) * ib;
    }
    gsync();
    int cur = 0;
    double xl = 0.0;
    bool solved = false;
    for (int dl = 1; dl < P; dl <<= 1) {
        if (act) {
            int im = p - dl, ip = p + dl;
            if (cyclic) {
                im = im < 0 ? im + P : im;
                ip = ip >= P ? ip - P : ip;
            } else {
                im = im < -1 ? -1 : im;
                ip = ip > P ? P : ip;
            }
            double li = F(cur, 0, p), ui = F(cur, 1, p), ri = F(cur, 2, p);
            const double lm = F(cur, 0, im), um = F(cur, 1, im), rm = F(cur, 2, im);
            const double lp = F(cur, 0, ip), up = F(cur, 1, ip), rp = F(cur, 2, ip);
            if (cyclic && 2 * dl == P) {
                const double si = li + ui, sj = lm + um;
                xl = (ri - si * rm) * rcp_nr(1.0 - si * sj);
                solved = true;
            } else {
                pcr_step(li, ui, ri, lm, um, rm, lp, up, rp);
                F(cur ^ 1, 0, p) = li;
                F(cur ^ 1, 1, p) = ui;
                F(cur ^ 1, 2, p) = ri;
            }
        }
        gsync();
        cur ^= 1;
    }
    if (act) {
        if (!solved) xl = F(cur, 2, p);
        F(cur ^ 1, 2, p) = xl;
    }
    gsync();
    double xlm = 0.0;
    if (act) {
        if (cyclic)
            xlm = F(cur ^ 1, 2, p == 0 ? P - 1 : p - 1);
        else
            xlm = p == 0 ? 0.0 : F(cur ^ 1, 2, p - 1);
    }
    const double xf = act ? r0 - l0 * xlm - u0 * xl : 0.0;
    if (!act) xl = 0.0;

    // ------------------------------------------------ back substitution
    double* xp = a.X + row0;
    double nonfinite = fma(xf, 0.0, fma(xl, 0.0, 0.0));
    double xn = xl;
    // staged: x overwrites delta in the D field (each row's delta is read just
    // before) and leaves coalesced
    auto XO = [&](int k) -> double& { return stt[2 * fs + SL(k)]; };
#pragma unroll
    for (int k = M - 2; k >= 1; --k) {
        if (k <= m - 2) {
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
            rag_locate(r, base, rem, inv0, inv1, q, k);
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
// inside it, with barriers of their own).  a.mcap must be RAG_MT.
constexpr int RAG_PERSIST_THREADS = 256;
constexpr int RAG_PERSIST_CLASSES = 3;
// shared-memory slice of a group of P threads (nested: two slices of P / 2
// fit in one of P)
__host__ __device__ __forceinline__ size_t rag_persist_slice(int P) {
    return rag_cta_smem_bytes(64, true, RAG_MT) * (size_t)(P / 64);
}
template <typename TIN>
__global__ void __launch_bounds__(RAG_PERSIST_THREADS, 2) ragged_persist_kernel(const RagArgs a) {
    extern __shared__ double rsm[];
    __shared__ int next_task[1 << RAG_PERSIST_CLASSES];  // by barrier id (unique per group)
    const int tid = threadIdx.x;
    for (int c = 0; c < RAG_PERSIST_CLASSES; ++c) {
        const int P = RAG_PERSIST_THREADS >> c;
        const int g = tid / P, p = tid % P;
        const int bid = (1 << c) + g;  // 1; 2, 3; 4 .. 7
        double* sm = rsm + rag_persist_slice(P) / sizeof(double) * g;
        for (;;) {
            if (p == 0) next_task[bid] = atomicAdd(&a.next[c], 1);
            asm volatile("bar.sync %0, %1;" ::"r"(bid), "r"(P) : "memory");
            const int t = next_task[bid];
            if (t >= a.cls_count[c]) break;
            const int4 task = a.tasks[a.cls_first[c] + t];
            if (task.w)
                rag_cta_body<TIN, true>(a, task, P, sm, p, bid);
            else
                rag_cta_body<TIN, false>(a, task, P, sm, p, bid);
            // the group's shared memory and next_task are rewritten by its next task
            asm volatile("bar.sync %0, %1;" ::"r"(bid), "r"(P) : "memory");
        }
    }
}

}  // namespace btdma
