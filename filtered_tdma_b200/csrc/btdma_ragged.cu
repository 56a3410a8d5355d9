// C ABI of ragged (CSR) batches: length buckets, task tables, launches on
// forked side streams, the autotuner (declared in include/btdma.h).
#include <algorithm>
#include <climits>

#include "btdma_host.cuh"
#include "k_ragged.cuh"

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

// Interleaved buckets (cta_per_system 3): the padded batch's rows and systems,
// and its scratch (gathered A, B, C, D of elem bytes, then x in FP64).
int rag_il_rows(const btdma_handle::RagBucket& b) { return (b.nmax + TILE_MT - 1) / TILE_MT * TILE_MT; }
int rag_il_cols(const btdma_handle::RagBucket& b) { return (b.count + 3) / 4 * 4; }
size_t rag_il_bytes(const btdma_handle::RagBucket& b, int elem) {
    const size_t plane = (size_t)rag_il_rows(b) * rag_il_cols(b);
    return plane * (4 * (size_t)elem + sizeof(double));
}
// Gives bucket b its scratch for the interleaved kind (kept with the plan).
int rag_il_alloc(btdma_handle::RagBucket& b, int elem) {
    cudaFree(b.ibuf);
    b.ibuf = nullptr;
    b.npad = rag_il_rows(b);
    b.nbp = rag_il_cols(b);
    CK(cudaMalloc(&b.ibuf, rag_il_bytes(b, elem)));
    return BTDMA_OK;
}
void rag_il_free(btdma_handle::RagBucket& b) {
    cudaFree(b.ibuf);
    b.ibuf = nullptr;
}

// One interleaved bucket: gather, tiled solve, scatter (stream order).  1 when
// solved, 0 when the tiled kernel does not take the padded shape, < 0 on error.
template <typename TIN>
int rag_il_run(btdma_t h, const btdma_handle::RagBucket& b, const TIN* A, const TIN* B,
               const TIN* C, const TIN* D, double* X, cudaStream_t st) {
    const int npad = b.npad, nbp = b.nbp;
    const size_t plane = (size_t)npad * nbp;
    TIN* g = static_cast<TIN*>(b.ibuf);
    double* xi = reinterpret_cast<double*>(g + 4 * plane);
    const dim3 blk(32, 8), grd((nbp + RAG_IL_TILE - 1) / RAG_IL_TILE,
                               (npad + RAG_IL_TILE - 1) / RAG_IL_TILE);
    rag_gather_kernel<TIN><<<grd, blk, 0, st>>>(A, B, C, D, h->rag_d_off, h->rag_d_list, b.first,
                                                b.count, npad, nbp, g);
    CK(cudaGetLastError());
    const int rc = tile_solve_batch(g, g + plane, g + 2 * plane, g + 3 * plane, (int)sizeof(TIN),
                                    xi, nbp, npad, h->status, st);
    if (rc <= 0) return rc;
    rag_scatter_kernel<<<grd, blk, 0, st>>>(xi, h->rag_d_off, h->rag_d_list, b.first, b.count,
                                            npad, nbp, X);
    CK(cudaGetLastError());
    return 1;
}

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

// Task tables of the whole plan: warp-kind launches (buckets longest first;
// one for the buckets of at most RAG_MT rows per lane and one for the longer
// ones, since a launch's shared memory is sized by its longest bucket and
// would otherwise halve the short buckets' occupancy), one persistent launch
// for every CTA-kind bucket of at most RAG_PERSIST_THREADS threads (tasks
// {list index, cyclic, P, staged}, the longest systems first) followed by the
// warp-kind buckets of at most RAG_MT rows per lane as its warp class (so the
// launch's tail is short work; those buckets then get no launch of their own),
// and one CTA-kind launch per longer P.
int rag_build_launches(btdma_t h) {
    std::vector<int4> tasks;
    h->rag_launches.clear();
    for (int longer = 0; longer < 2; ++longer) {
        btdma_handle::RagLaunch wl{0, 0, (int)tasks.size(), 0, 1, 0};
        if (!longer && h->rag_persist) continue;  // the persistent launch's warp class
        for (int i = (int)h->rag_buckets.size() - 1; i >= 0; --i) {
            const auto& b = h->rag_buckets[i];
            if (b.inter || b.cta || (rag_mcap(b.nmax, b.P) > RAG_MT) != (longer != 0)) continue;
            rag_bucket_tasks(b, 0, b.P, tasks);
            wl.mcap = std::max(wl.mcap, rag_mcap(b.nmax, b.P));
        }
        wl.count = (int)tasks.size() - wl.first;
        if (wl.count) h->rag_launches.push_back(wl);
    }
    if (h->rag_persist) {
        // one class per P (256, 128, 64), each longest first
        btdma_handle::RagLaunch pl{2, RAG_PERSIST_THREADS, (int)tasks.size(), 0, RAG_MT, 0};
        for (int c = 0; c < RAG_PERSIST_CLASSES; ++c) {
            const int Pc = RAG_PERSIST_THREADS >> c;
            std::vector<int> ids;
            for (int i = 0; i < (int)h->rag_buckets.size(); ++i)
                if (!h->rag_buckets[i].inter && h->rag_buckets[i].cta &&
                    h->rag_buckets[i].P == Pc)
                    ids.push_back(i);
            std::stable_sort(ids.begin(), ids.end(), [&](int x, int y) {
                return h->rag_buckets[x].nmax > h->rag_buckets[y].nmax;
            });
            h->rag_cls_first[c] = (int)tasks.size() - pl.first;
            for (int i : ids) {
                const auto& b = h->rag_buckets[i];
                for (int k = 0; k < b.count; ++k)
                    tasks.push_back(make_int4(b.first + k, b.cyc, b.P, b.staged));
            }
            h->rag_cls_count[c] = (int)tasks.size() - pl.first - h->rag_cls_first[c];
        }
        // warp class: warp-kind buckets of at most RAG_MT rows a lane, longest first
        h->rag_warp_first = (int)tasks.size() - pl.first;
        for (int i = (int)h->rag_buckets.size() - 1; i >= 0; --i) {
            const auto& b = h->rag_buckets[i];
            if (b.inter || b.cta || rag_mcap(b.nmax, b.P) > RAG_MT) continue;
            rag_bucket_tasks(b, 0, b.P, tasks);
        }
        h->rag_warp_count = (int)tasks.size() - pl.first - h->rag_warp_first;
        pl.count = (int)tasks.size() - pl.first;
        if (pl.count) h->rag_launches.push_back(pl);
    }
    for (int P = 512; P >= 64; P >>= 1) {
        if (h->rag_persist && P <= RAG_PERSIST_THREADS) break;
        for (int stg = 0; stg < 2; ++stg) {
            btdma_handle::RagLaunch cl{1, P, (int)tasks.size(), 0, 1, stg};
            for (const auto& b : h->rag_buckets)
                if (!b.inter && b.cta && b.P == P && b.staged == stg) {
                    rag_bucket_tasks(b, 1, P, tasks);
                    cl.mcap = std::max(cl.mcap, rag_mcap(b.nmax, P));
                }
            cl.count = (int)tasks.size() - cl.first;
            if (cl.count) h->rag_launches.push_back(cl);
        }
    }
    // interleaved buckets: a launch sequence each (cta 3, P = the bucket's index)
    for (int i = 0; i < (int)h->rag_buckets.size(); ++i)
        if (h->rag_buckets[i].inter)
            h->rag_launches.push_back(btdma_handle::RagLaunch{3, i, 0, 0, 0, 0});
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
    for (auto& b : h->rag_buckets) rag_il_free(b);
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
    if (!h->rag_d_next) CK(cudaMalloc(&h->rag_d_next, sizeof(int) * (RAG_PERSIST_CLASSES + 1)));
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
    a.next = h->rag_d_next;
    if (cta == 2) {
        auto kern = ragged_persist_kernel<TIN>;
        const size_t smem = rag_persist_slice(RAG_PERSIST_THREADS);
        for (int c = 0; c < RAG_PERSIST_CLASSES; ++c) {
            a.cls_first[c] = h->rag_cls_first[c];
            a.cls_count[c] = h->rag_cls_count[c];
        }
        a.warp_first = h->rag_warp_first;
        a.warp_count = h->rag_warp_count;
        static bool attr_done = false;
        static int per_sm = 1;
        if (!attr_done) {
            CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, RAG_PERSIST_THREADS,
                                                             smem));
            per_sm = std::max(1, per_sm);
            attr_done = true;
        }
        a.mcap = RAG_MT;
        CK(cudaMemsetAsync(h->rag_d_next, 0, sizeof(int) * (RAG_PERSIST_CLASSES + 1), st));
        kern<<<std::min(n_tasks, per_sm * num_sms()), RAG_PERSIST_THREADS, smem, st>>>(a);
    } else if (cta) {
        if (staged && rag_cta_smem_bytes(P, true, mcap) > (size_t)max_smem_optin()) staged = 0;
        auto kern = staged ? ragged_cta_kernel<TIN, true> : ragged_cta_kernel<TIN, false>;
        static bool attr_done[2] = {false, false};
        if (!attr_done[staged]) {
            CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    max_smem_optin()));
            attr_done[staged] = true;
        }
        const size_t smem = rag_cta_smem_bytes(P, staged, mcap);
        // co-resident CTAs of this shape (cached per shape): the prefetch distance
        static int resident[2][4][RAG_MT + 1] = {};
        const int pi = P == 64 ? 0 : P == 128 ? 1 : P == 256 ? 2 : 3;
        int& res = resident[staged][pi][std::min(std::max(mcap, 0), RAG_MT)];
        if (res == 0) {
            int per_sm = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, P, smem));
            res = std::max(1, per_sm) * num_sms();
        }
        a.pf_ahead = res;
        kern<<<n_tasks, P, smem, st>>>(a);
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
        if (L[i].cta == 3) {
            const int rc = rag_il_run<TIN>(h, h->rag_buckets[L[i].P], A, B, C, D, X, s);
            if (rc < 0) return rc;
            if (rc == 0) return fail(BTDMA_ERR_UNSUPPORTED, "interleaved bucket not tileable");
            continue;
        }
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
            int cta, P, staged;  // cta 3: interleaved
        };
        std::vector<Cand> cands;
        if (!b.cyc) cands.push_back({3, 1, 0});
        for (int P = 1; P <= 32 && b.nmin / P >= 3; P <<= 1)
            if (rag_mcap(b.nmax, P) <= RAG_WARP_MCAP) cands.push_back({0, P, 0});
        for (int P = 64; P <= 512 && b.nmin / P >= 3; P <<= 1)
            if (rag_mcap(b.nmax, P) <= RAG_MT) {
                cands.push_back({1, P, 0});
                if (rag_cta_smem_bytes(P, true, rag_mcap(b.nmax, P)) <=
                    (size_t)max_smem_optin())
                    cands.push_back({1, P, 1});
            }
        float best = 1e30f;
        Cand pick{b.inter ? 3 : b.cta, b.P, b.staged};
        for (const Cand& cd : cands) {
            if (cd.cta == 3) {  // gather + tiled solve + scatter, on its own scratch
                if ((rc = rag_il_alloc(b, (int)sizeof(TIN)))) break;
                float ms = 0.f;
                int ran = 1;
                for (int rep = 0; rep < 3 && !rc && ran == 1; ++rep) {
                    CK(cudaEventRecord(e0, st));
                    ran = rag_il_run<TIN>(h, b, A, B, C, D, X, st);
                    if (ran < 0) rc = ran;
                    if (ran != 1) break;
                    CK(cudaEventRecord(e1, st));
                    CK(cudaEventSynchronize(e1));
                    float t = 0.f;
                    CK(cudaEventElapsedTime(&t, e0, e1));
                    ms = rep == 0 ? t : std::min(ms, t);
                }
                if (rc) break;
                if (ran == 1 && ms < best) {
                    best = ms;
                    pick = cd;
                }
                continue;
            }
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
        b.inter = pick.cta == 3;
        if (!b.inter) rag_il_free(b);
        b.cta = pick.cta == 3 ? 0 : pick.cta;
        b.staged = pick.staged;
        b.P = pick.P;
        b.warps = pick.cta ? pick.P / 32 : RAG_WPC;
        b.mcap = rag_mcap(b.nmax, pick.P);
        b.best_ms = best;
    }
    // the whole plan: the launch structure (a launch per CTA-kind shape, or the
    // persistent launch) crossed with the CTA-kind buckets' staging as tuned
    // bucket by bucket, all staged (where the staged tile fits) or all
    // unstaged -- buckets timed alone do not see how they share the GPU in the
    // solve; each plan timed as a whole (best of 3 after a warm-up), the
    // fastest kept
    std::vector<int> tuned_staged;
    for (const auto& b : h->rag_buckets) tuned_staged.push_back(b.staged);
    auto apply = [&](int mode) {  // 0: as tuned, 1: all staged, 2: all unstaged
        for (size_t i = 0; i < h->rag_buckets.size(); ++i) {
            auto& b = h->rag_buckets[i];
            if (!b.cta || b.inter) continue;
            b.staged = mode == 0 ? tuned_staged[i]
                       : mode == 2 ? 0
                                   : (rag_cta_smem_bytes(b.P, true, b.mcap) <=
                                      (size_t)max_smem_optin());
        }
    };
    float best_whole = 1e30f;
    int best_mode = 0, best_pers = 0;
    for (int mode = 0; mode < 3 && !rc; ++mode) {
        apply(mode);
        for (int pers = 0; pers < 2 && !rc; ++pers) {
            h->rag_persist = pers != 0;
            if ((rc = rag_build_launches(h))) break;
            float whole = 1e30f;
            for (int rep = 0; rep < 4 && !rc; ++rep) {
                CK(cudaEventRecord(e0, st));
                rc = rag_run<TIN>(h, A, B, C, D, X, st);
                if (rc) break;
                CK(cudaEventRecord(e1, st));
                CK(cudaEventSynchronize(e1));
                float t = 0.f;
                CK(cudaEventElapsedTime(&t, e0, e1));
                if (rep > 0) whole = std::min(whole, t);  // rep 0 warms up
            }
            if (whole < best_whole) {
                best_whole = whole;
                best_mode = mode;
                best_pers = pers;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    apply(best_mode);
    h->rag_persist = best_pers != 0;
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

int btdma_ragged_set_plan(btdma_t h, const btdma_ragged_bucket* in, int n) {
    if (!h || (!in && n > 0)) return fail(BTDMA_ERR_ARG, "null argument");
    if (n != (int)h->rag_buckets.size())
        return fail(BTDMA_ERR_ARG, "the current plan has %d buckets, %d given",
                    (int)h->rag_buckets.size(), n);
    for (int i = 0; i < n; ++i) {
        const auto& b = h->rag_buckets[i];
        const btdma_ragged_bucket& g = in[i];
        if (g.periodic != b.cyc || g.n_systems != b.count || g.n_row_min != b.nmin ||
            g.n_row_max != b.nmax)
            return fail(BTDMA_ERR_ARG, "bucket %d does not match the current plan", i);
        const int P = g.lanes_per_system, kind = g.cta_per_system;
        if (P <= 0 || (P & (P - 1)) != 0 || b.nmin / P < 3)
            return fail(BTDMA_ERR_ARG, "bucket %d: %d lanes per system", i, P);
        if (kind == 0) {
            if (P > 32 || rag_mcap(b.nmax, P) > RAG_WARP_MCAP)
                return fail(BTDMA_ERR_ARG, "bucket %d: warp kind needs P <= 32 and <= %d rows "
                            "per lane", i, RAG_WARP_MCAP);
        } else if (kind == 3) {
            if (b.cyc)
                return fail(BTDMA_ERR_ARG, "bucket %d: periodic systems cannot be padded into an "
                            "interleaved batch", i);
            if (tile_plan(rag_il_rows(b), false, h->precision == BTDMA_FP64 ? 8 : 4).sys == 0)
                return fail(BTDMA_ERR_ARG, "bucket %d: the tiled kernel does not take %d rows", i,
                            rag_il_rows(b));
        } else if (kind == 1 || kind == 2) {
            if (P < 64 || P > 512 || rag_mcap(b.nmax, P) > RAG_MT)
                return fail(BTDMA_ERR_ARG, "bucket %d: CTA kind needs 64 <= P <= 512 and <= %d "
                            "rows per thread", i, RAG_MT);
            if (kind == 2 &&
                rag_cta_smem_bytes(P, true, rag_mcap(b.nmax, P)) > (size_t)max_smem_optin())
                return fail(BTDMA_ERR_ARG, "bucket %d: a staged system of %d threads does not "
                            "fit in shared memory", i, P);
        } else {
            return fail(BTDMA_ERR_ARG, "bucket %d: cta_per_system %d", i, kind);
        }
    }
    for (int i = 0; i < n; ++i) {
        auto& b = h->rag_buckets[i];
        b.P = in[i].lanes_per_system;
        b.inter = in[i].cta_per_system == 3 ? 1 : 0;
        b.cta = in[i].cta_per_system == 1 || in[i].cta_per_system == 2 ? 1 : 0;
        b.staged = in[i].cta_per_system == 2 ? 1 : 0;
        if (b.inter) {
            const int rc = rag_il_alloc(b, h->precision == BTDMA_FP64 ? 8 : 4);
            if (rc) return rc;
        } else {
            rag_il_free(b);
        }
        b.warps = b.cta ? b.P / 32 : RAG_WPC;
        b.mcap = rag_mcap(b.nmax, b.P);
        b.best_ms = in[i].tuned_ms;
    }
    // the persistent launch when any bucket is marked for it
    h->rag_persist = false;
    for (int i = 0; i < n; ++i) h->rag_persist |= in[i].persistent != 0;
    return rag_build_launches(h);
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
        out[i].cta_per_system = b.inter ? 3 : b.cta + b.staged;
        out[i].tuned_ms = b.best_ms;
        out[i].persistent = h->rag_persist && !b.inter &&
                                    (b.cta ? b.P <= RAG_PERSIST_THREADS
                                           : rag_mcap(b.nmax, b.P) <= RAG_MT)
                                ? 1
                                : 0;
    }
    return BTDMA_OK;
}
