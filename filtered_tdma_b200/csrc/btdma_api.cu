// C ABI of the batched tridiagonal library (declared in include/btdma.h): handle
// life cycle, uniform-batch solves (serial Thomas, tiled PaScaL, reference-order
// segment kernels, Filtered v1/v2), FP32 storage and refinement, the
// allocation-free entry point and the self test.  The handle owns every device
// buffer a solve needs (allocated once in btdma_create), so solves allocate
// nothing and can be captured in CUDA graphs.  Ragged batches live in
// btdma_ragged.cu, the application steps (heat, channel Poisson, momentum) in
// btdma_apps.cu; the shared host machinery in btdma_host.cuh.
#include <cstdarg>
#include <mutex>

#include "btdma_host.cuh"
#include "k_filtered_j.cuh"
#include "k_refine.cuh"
#include "k_thomas.cuh"

namespace btdma_host {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

}  // namespace btdma_host

int tile_solve_batch(const void* A, const void* B, const void* C, const void* D, int elem,
                     double* X, int n_sys, int n_row, unsigned* status, cudaStream_t st) {
    if (elem == 8)
        return try_tile<double>(static_cast<const double*>(A), static_cast<const double*>(B),
                                static_cast<const double*>(C), static_cast<const double*>(D), X,
                                n_sys, n_row, false, status, st, false, nullptr,
                                BTDMA_TILE_AUTO);
    return try_tile<float>(static_cast<const float*>(A), static_cast<const float*>(B),
                           static_cast<const float*>(C), static_cast<const float*>(D), X, n_sys,
                           n_row, false, status, st, false, nullptr, BTDMA_TILE_AUTO);
}

namespace {

int jmax_launch(btdma_t h, const double* D, int n_sys, int n_row, cudaStream_t st) {
    int blocks = std::max(1, std::min((n_sys + JRED_BLOCK - 1) / JRED_BLOCK, 1184 / h->P + 1));
    jmax_kernel<<<dim3(blocks, h->P), JRED_BLOCK, 0, st>>>(
        D, n_sys, n_row, h->P, (h->flags & BTDMA_FLAG_J_HOST) ? 1 : 0, h->work);
    CK(cudaGetLastError());
    return BTDMA_OK;
}

// exact: the device word jfinal sets when the batch needs the exact reduced
// solve (null: the reference's behaviour, no fallback)
int jfinal_launch(btdma_t h, int n_row, int version, unsigned* exact, cudaStream_t st) {
    jfinal_kernel<<<1, 32, 0, st>>>(h->work, h->J, h->rho_row, n_row, h->P, h->eps_constant,
                                    version, (h->flags & BTDMA_FLAG_J_HOST) ? 1 : 0, exact);
    CK(cudaGetLastError());
    return BTDMA_OK;
}

// Sub-segments per Filtered segment when the tiled kernels take a Filtered
// batch of P segments: R = n_row / (16 P), a power of two, with at most 32
// sub-segments a system (a power of two when periodic); 0 when they do not.
int filtered_tile_lanes(int n_row, int P, bool cyclic) {
    if (P < 2 || n_row % TILE_MT != 0) return 0;
    const int nseg = n_row / TILE_MT;
    if (nseg > 32 || nseg % P != 0) return 0;
    const int R = nseg / P;
    if ((R & (R - 1)) != 0) return 0;
    if (cyclic && (nseg & (nseg - 1)) != 0) return 0;
    return R;
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
    h->last_n_sys = n_sys;
    h->last_refined = false;
    h->last_filtered = false;

    if (h->P == 1) {
        if (cyclic && n_row < 3) return fail(BTDMA_ERR_ARG, "periodic systems need n_row >= 3");
        // short systems: c' and d' stay in shared memory (40 B/row).  Measured on
        // B200 against thomas_f64_kernel (c', d' through HBM, 72 B/row): faster
        // up to 64 rows at every batch size (4096 x 64: 33 vs 47 us; 262144 x
        // 64: 182 vs 191 us), and up to 128 rows for batches of at most 2^21
        // rows (4096 x 128: 43 vs 70 us); slower for large 128-row batches (at
        // most 3 one-warp CTAs fit an SM: 262144 x 128, 472 vs 374 us).
        const bool staged = n_row <= 64 || (n_row <= THOMAS_STAGED_MAX_ROWS &&
                                            (long long)n_sys * n_row <= (1ll << 21));
        if (!cyclic && staged && tma_ok(C, n_sys) && tma_ok(D, n_sys) && tma_ok(X, n_sys)) {
            CUtensorMap mc, md, mx;
            if (make_map(&mc, C, n_sys, n_row) && make_map(&md, D, n_sys, n_row) &&
                make_map(&mx, X, n_sys, n_row)) {
                static bool attr_done = false;
                if (!attr_done) {
                    CK(cudaFuncSetAttribute(
                        thomas_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                        (int)thomas_staged_smem_bytes(THOMAS_STAGED_MAX_ROWS)));
                    attr_done = true;
                }
                const int grid = (n_sys + THOMAS_STAGED_SYS - 1) / THOMAS_STAGED_SYS;
                thomas_staged_kernel<<<grid, THOMAS_STAGED_SYS, thomas_staged_smem_bytes(n_row),
                                       st>>>(mc, md, mx, A, B, n_sys, n_row, h->status);
                CK(cudaGetLastError());
                return BTDMA_OK;
            }
        }
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
        rc = try_tile<double>(A, B, C, D, X, n_sys, n_row, cyclic, h->status, st, false,
                              nullptr, h->tile_shape);
        if (rc < 0) return rc;
        if (rc == 1) return BTDMA_OK;
    }

    // Filtered v2 on the tiled kernels: the reference's P segments are groups
    // of R = n_row / (16 P) sub-segments of the tiled solve, whose reduced
    // system takes Filtered's 2 x 2 interfaces (reduced_solve_filtered).  J
    // and the exact-fallback word come from the reference's device estimator
    // as below; the Filtered launch runs while the word is 0, the exact tiled
    // PaScaL while it is set.  Shapes the tiled kernels do not take go to the
    // segment kernels below (the J accumulators reset themselves).
    if (h->method == BTDMA_FILTERED_V2 && !(h->flags & BTDMA_FLAG_REFERENCE_ORDER)) {
        const int R = filtered_tile_lanes(n_row, h->P, cyclic);
        if (R > 0) {
            if ((rc = jmax_launch(h, D, n_sys, n_row, st))) return rc;
            if ((rc = jfinal_launch(h, n_row, 2, h->exact, st))) return rc;
            rc = try_tile<double>(A, B, C, D, X, n_sys, n_row, cyclic, h->status, st, false,
                                  h->exact, h->tile_shape, R, true);
            if (rc < 0) return rc;
            if (rc == 1) {
                h->last_filtered = true;
                rc = try_tile<double>(A, B, C, D, X, n_sys, n_row, cyclic, h->status, st, false,
                                      h->exact, h->tile_shape);
                if (rc < 0) return rc;
                if (rc == 1) return BTDMA_OK;
                return fail(BTDMA_ERR_UNSUPPORTED, "exact fallback not tileable");
            }
        }
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
    if (seg_smem_bytes(a.mcap, a.P, cyclic, h->method == BTDMA_PASCAL,
                       seg_reg_rows(n_row, a.P)) > (size_t)max_smem_optin())
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

    if (h->method == BTDMA_PASCAL)
        return cyclic ? launch_seg_method<true>(h->method, maps, a, groups, st)
                      : launch_seg_method<false>(h->method, maps, a, groups, st);

    // Filtered.  Unless the reference's behaviour is asked for, a batch whose J
    // reaches m - 2 (or whose rho is >= 0.5) in some segment takes the exact
    // reduced solve instead: jfinal sets the device word h->exact, the
    // Filtered kernel runs only while it is 0 and the exact solve only while it
    // is 1 (both launched; no host round trip).
    unsigned* exact = (h->flags & BTDMA_FLAG_REFERENCE_ORDER) ? nullptr : h->exact;
    if (h->method == BTDMA_FILTERED_V2) {
        if ((rc = jmax_launch(h, D, n_sys, n_row, st))) return rc;
        if ((rc = jfinal_launch(h, n_row, 2, exact, st))) return rc;
    } else {
        SegArgs ai = a;
        ai.mode = SEG_MODE_INTERFACE;
        rc = cyclic ? launch_seg_method<true>(h->method, maps, ai, groups, st)
                    : launch_seg_method<false>(h->method, maps, ai, groups, st);
        if (rc) return rc;
        if ((rc = jfinal_launch(h, n_row, 1, exact, st))) return rc;
    }
    h->last_filtered = true;
    a.gate = exact;
    a.gate_run = 0;
    rc = cyclic ? launch_seg_method<true>(h->method, maps, a, groups, st)
                : launch_seg_method<false>(h->method, maps, a, groups, st);
    if (rc || !exact) return rc;
    // the exact solve: the tiled PaScaL kernel, or the reference-order one
    // where the shape is not tiled
    rc = try_tile<double>(A, B, C, D, X, n_sys, n_row, cyclic, h->status, st, false, exact,
                          h->tile_shape);
    if (rc < 0) return rc;
    if (rc == 1) return BTDMA_OK;
    if (seg_smem_bytes(a.mcap, a.P, cyclic, true, seg_reg_rows(n_row, a.P)) >
        (size_t)max_smem_optin())
        return fail(BTDMA_ERR_UNSUPPORTED,
                    "segment of %d rows does not fit in shared memory for the exact fallback",
                    a.mcap);
    a.gate_run = 1;
    return cyclic ? launch_seg_method<true>(BTDMA_PASCAL, maps, a, groups, st)
                  : launch_seg_method<false>(BTDMA_PASCAL, maps, a, groups, st);
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
    CKC(cudaMalloc(&h->exact, sizeof(unsigned)));
    CKC(cudaMemset(h->exact, 0, sizeof(unsigned)));
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
    for (auto& b : h->rag_buckets) cudaFree(b.ibuf);
    cudaFree(h->rho_row);
    cudaFree(h->J);
    cudaFree(h->work);
    cudaFree(h->status);
    cudaFree(h->exact);
    cudaFree(h->scratch);
    cudaFree(h->resid);
    cudaFree(h->iters);
    cudaFree(h->open);
    cudaFree(h->rag_d_off);
    cudaFree(h->rag_d_list);
    cudaFree(h->rag_d_tasks);
    cudaFree(h->rag_d_probe);
    cudaFree(h->rag_d_next);
    for (int i = 0; i < btdma_handle::RAG_STREAMS; ++i) {
        if (h->rag_side[i]) cudaStreamDestroy(h->rag_side[i]);
        if (h->rag_join[i]) cudaEventDestroy(h->rag_join[i]);
    }
    if (h->rag_fork) cudaEventDestroy(h->rag_fork);
    if (auto* p = h->hp) {
        cudaFree(p->buf);
        for (auto s : p->s)
            if (s) cudaStreamDestroy(s);
        for (auto e : {p->start, p->done, p->in[0], p->in[1], p->solved[0], p->solved[1],
                       p->out[0], p->out[1]})
            if (e) cudaEventDestroy(e);
        delete p;
    }
    delete h;
    return BTDMA_OK;
}

// Host-buffer solve: the batch passes through the GPU in chunks of systems,
// each gathered from the [n_row][n_sys] host arrays by a 2-D copy into a
// contiguous [n_row][chunk] device buffer; with two buffer sets, the copy-in
// of chunk i + 1 (one copy engine), the solve of chunk i and the copy-out of
// chunk i - 1 (the other copy engine) overlap.  Systems are independent, so a
// PaScaL chunk solves exactly as in a whole-batch call; a Filtered batch goes
// through as one chunk, its truncation depth depending on the whole batch's
// right-hand sides.
int btdma_solve_host(btdma_t h, const double* hA, const double* hB, const double* hC,
                     const double* hD, double* hX, int n_sys, int n_row, int cyclic,
                     cudaStream_t stream) {
    int rc = check_sizes(h, n_sys, n_row);
    if (rc) return rc;
    if (!hA || !hB || !hC || !hD || !hX) return fail(BTDMA_ERR_ARG, "null array");
    if (h->precision != BTDMA_FP64)
        return fail(BTDMA_ERR_UNSUPPORTED, "host-buffer solves need an FP64 handle");
    // 16 chunks: the pipeline's unoverlapped ends (the first copy-in, the last
    // solve and copy-out) are one chunk each; measured 81.9 ms against 82.5 ms
    // at 8 and 82.2 ms at 32 for 262144 x 512
    constexpr int CHUNKS = 16, MIN_CHUNK = 4096;
    int chunk = n_sys;
    if (h->method == BTDMA_PASCAL) {
        chunk = ((n_sys + CHUNKS - 1) / CHUNKS + 31) / 32 * 32;
        chunk = std::min(std::max(chunk, MIN_CHUNK), n_sys);
    }
    const size_t ce = ((size_t)chunk * n_row + 31) / 32 * 32;  // 256-byte aligned arrays
    auto* p = h->hp;
    if (!p) {
        p = h->hp = new btdma_handle::HostPipe;
        for (auto& s : p->s) CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        for (auto* e : {&p->start, &p->done, &p->in[0], &p->in[1], &p->solved[0],
                        &p->solved[1], &p->out[0], &p->out[1]})
            CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    if (p->chunk_elems < ce) {
        CK(cudaStreamSynchronize(p->s[2]));  // the previous call's copies are done
        CK(cudaFree(p->buf));
        p->buf = nullptr;
        p->chunk_elems = 0;
        CK(cudaMalloc(&p->buf, sizeof(double) * 10 * ce));
        p->chunk_elems = ce;
    }
    const size_t be = p->chunk_elems;  // elements per array of a buffer set
    const double* hin[4] = {hA, hB, hC, hD};
    const size_t pitch = sizeof(double) * (size_t)n_sys;
    // after the caller's earlier work on `stream`, and after this handle's
    // previous host-buffer solve (its buffers are reused)
    CK(cudaEventRecord(p->start, stream));
    for (auto s : p->s) {
        CK(cudaStreamWaitEvent(s, p->start, 0));
        CK(cudaStreamWaitEvent(s, p->done, 0));
    }
    const int nch = (n_sys + chunk - 1) / chunk;
    for (int i = 0; i < nch; ++i) {
        const int b = i & 1, s0 = i * chunk, c = std::min(chunk, n_sys - s0);
        double* d = p->buf + (size_t)b * 5 * be;  // A, B, C, D, X of buffer set b
        const size_t w = sizeof(double) * (size_t)c;
        if (i >= 2) CK(cudaStreamWaitEvent(p->s[0], p->solved[b], 0));
        for (int k = 0; k < 4; ++k)
            CK(cudaMemcpy2DAsync(d + k * be, w, hin[k] + s0, pitch, w, n_row,
                                 cudaMemcpyHostToDevice, p->s[0]));
        CK(cudaEventRecord(p->in[b], p->s[0]));
        CK(cudaStreamWaitEvent(p->s[1], p->in[b], 0));
        if (i >= 2) CK(cudaStreamWaitEvent(p->s[1], p->out[b], 0));
        if ((rc = solve_impl(h, d, d + be, d + 2 * be, d + 3 * be, d + 4 * be, c, n_row,
                             cyclic != 0, p->s[1]))) {
            // copies already queued still reference the host arrays: order the
            // caller's stream after them before reporting the error
            const std::string msg = g_err;
            if (cudaEventRecord(p->done, p->s[2]) == cudaSuccess &&
                cudaStreamWaitEvent(p->s[0], p->done, 0) == cudaSuccess &&
                cudaEventRecord(p->done, p->s[0]) == cudaSuccess)
                cudaStreamWaitEvent(stream, p->done, 0);
            h->last_stream = stream;
            g_err = msg;
            return rc;
        }
        CK(cudaEventRecord(p->solved[b], p->s[1]));
        CK(cudaStreamWaitEvent(p->s[2], p->solved[b], 0));
        CK(cudaMemcpy2DAsync(hX + s0, pitch, d + 4 * be, w, w, n_row, cudaMemcpyDeviceToHost,
                             p->s[2]));
        CK(cudaEventRecord(p->out[b], p->s[2]));
    }
    CK(cudaEventRecord(p->done, p->s[2]));
    CK(cudaStreamWaitEvent(stream, p->done, 0));
    h->last_stream = stream;
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
    h->last_filtered = false;
    const bool cyc = cyclic != 0;
    const char* shape_msg =
        "FP32 storage needs n_row % 16 == 0, n_sys % 4 == 0, 16-byte alignment "
        "(and a power-of-two n_row/16 when periodic)";
    if (h->precision == BTDMA_FP32_STORE) {
        rc = try_tile<float>(A, B, C, D, X, n_sys, n_row, cyc, h->status, stream, false,
                             nullptr, h->tile_shape);
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
    st->filtered_exact = -1;
    if (h->last_filtered) {
        if (h->flags & BTDMA_FLAG_REFERENCE_ORDER) {
            st->filtered_exact = 0;
        } else {
            unsigned ex = 0;
            CK(cudaMemcpyAsync(&ex, h->exact, sizeof ex, cudaMemcpyDeviceToHost,
                               h->last_stream));
            CK(cudaStreamSynchronize(h->last_stream));
            st->filtered_exact = ex ? 1 : 0;
        }
    }
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

int btdma_set_tile_shape(btdma_t h, int shape) {
    if (!h) return fail(BTDMA_ERR_ARG, "null handle");
    if (shape < BTDMA_TILE_AUTO || shape > BTDMA_TILE_WIDE)
        return fail(BTDMA_ERR_ARG, "unknown tile shape %d", shape);
    h->tile_shape = shape;
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
// stand-in symbol), so its device address is looked up with the device
// current and cached per device, keyed on the CUDA context it was looked up
// in: a context that was destroyed and created again (cudaDeviceReset, a
// primary context released and retained) has its module loaded anew, so the
// address is looked up again there.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_noalloc_scratch[BTDMA_NOALLOC_MAX_ELEMS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
struct NoallocEntry {
    double* ptr = nullptr;
    unsigned long long ctx = 0;  // id of the context the address belongs to
    bool keyed = false;          // false: no context id available, look up every call
};
NoallocEntry g_noalloc[kMaxDevices];

// Unique id of the calling thread's current context (cuCtxGetId, through the
// runtime's driver entry points); false when there is none or the driver
// lacks the call.
bool current_ctx_id(unsigned long long* id) {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(p);
    });
    if (!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

int noalloc_scratch(double** out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(BTDMA_ERR_UNSUPPORTED, "device %d", dev);
    unsigned long long id = 0;
    bool have_id = current_ctx_id(&id);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocEntry& e = g_noalloc[dev];
    if (!e.ptr || !e.keyed || !have_id || e.ctx != id) {
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));  // creates the context if needed
        if (!have_id) have_id = current_ctx_id(&id);
        e.ptr = static_cast<double*>(p);
        e.ctx = have_id ? id : 0;
        e.keyed = have_id;
    }
    *out = e.ptr;
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
    if (threadIdx.x == 0) {
        (void)mbar_wait_bounded(&bar, 0, &status[0], limit);
        (void)mbar_wait_bounded_spin(&bar, 0, &status[1], limit);
    }
}

}  // namespace

int btdma_selftest_wait_timeout(int limit, unsigned* status_out, cudaStream_t stream) {
    if (limit <= 0 || limit > (1 << 16) || !status_out)
        return fail(BTDMA_ERR_ARG, "limit in [1, 65536] and an output word are required");
    unsigned* d = nullptr;
    CK(cudaMalloc(&d, 2 * sizeof(unsigned)));
    unsigned h[2] = {0, 0};
    cudaError_t e = cudaMemsetAsync(d, 0, 2 * sizeof(unsigned), stream);
    if (e == cudaSuccess) {
        selftest_wait_kernel<<<1, 32, 0, stream>>>(d, (uint32_t)limit);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    CK(e);
    *status_out = h[0] & h[1];  // a bit only if both waits raised it
    return BTDMA_OK;
}
