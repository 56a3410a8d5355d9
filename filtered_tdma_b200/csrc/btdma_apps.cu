// C ABI of the application steps built on the tiled solve with generated
// coefficients: the fused heat ADI step, the channel Poisson wall-normal
// solve and the channel momentum ADI sweeps (declared in include/btdma.h).
#include <cmath>
#include <cstring>

#include "btdma_host.cuh"
#include "k_heat.cuh"
#include "k_momentum.cuh"

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
    double* hpar = nullptr;  // {bx, by, dt 3 pi^2, iy, iz} for the fused Z sweep
    double* scratch = nullptr;  // full grid, the warm-up step before graph capture
    double* tab = nullptr;      // factor tables of the Z, Y, X sweeps, tab_stride apart
    size_t tab_stride = 0;      // (built once at create: the matrices are fixed)
    unsigned* status = nullptr;
    cudaStream_t cap = nullptr;  // private stream the step graph is captured on
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    double* graph_theta = nullptr;  // theta the graph was captured for
    cudaStream_t last_stream = nullptr;
};

namespace {

// One step as a kernel sequence on stream st (no host sync): right-hand side,
// then per direction a solve with generated coefficients and the re-layout
// for the next direction.  ev (optional): 8 events recorded around the phases
// (the profiled step).
int heat_enqueue(btdma_heat_t h, double* theta, cudaStream_t st, cudaEvent_t* ev = nullptr) {
    const HeatGeom& g = h->g;
    auto mark = [&](int i) {
        if (ev) cudaEventRecord(ev[i], st);
    };
    // constant-coefficient sweep of D into X, stored through the layout map
    // (xblk, xbs, xss, xrs) of the tiled solve (xblk = 0: X in D's layout)
    auto sweep = [&](int dir, const double* D, double* X, int n_sys, int n_row, double base,
                     int xblk, int xbs, int xss, int xrs, const char* name) {
        TileArgs ga = {};
        ga.cs = base;
        ga.cbound = 1;
        ga.xblk = xblk;
        ga.xbs = xbs;
        ga.xss = xss;
        ga.xrs = xrs;
        const int rc = try_tile_gen<1>(D, X, n_sys, n_row, ga, h->status, st,
                                       h->tab + dir * h->tab_stride, true);
        return rc == 1 ? BTDMA_OK
                       : (rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "%s sweep not tileable", name));
    };
    const dim3 b1(128, 1, 1), gr((g.ix + 127) / 128, g.iy, g.iz), bt(HEAT_TILE, 8, 1);
    const int tx = (g.ix + HEAT_TILE - 1) / HEAT_TILE, ty = (g.iy + HEAT_TILE - 1) / HEAT_TILE;
    int rc;
    mark(0);
    if (tile_plan_heat_z(g.iz).sys != 0) {
        // Z sweep with the right-hand side computed inside the solve from
        // theta (no right-hand-side pass); system jj * ix + ii, row kk;
        // solution to [jj][kk][ii]
        mark(1);
        TileArgs za = {};
        za.cs = g.bz;
        za.cbound = 1;
        za.xblk = g.ix;
        za.xbs = g.iz * g.ix;
        za.xss = 1;
        za.xrs = g.ix;
        za.ga = h->cosx;
        za.gb = h->cosy;
        za.gc = h->cosz;
        za.glam = h->hpar;
        rc = try_heat_z(theta, h->buf1, g.ix, g.iy, g.iz, za, h->status, st, h->tab);
        if (rc != 1) return rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "Z sweep not tileable");
    } else {
        heat_rhs_z_kernel<<<dim3((g.ix + 127) / 128, g.iy, (g.iz + HEAT_KCH - 1) / HEAT_KCH), b1,
                            0, st>>>(theta, h->buf0, g);
        CK(cudaGetLastError());
        mark(1);
        // Z sweep: system jj * ix + ii, row kk; solution to [jj][kk][ii]
        if ((rc = sweep(0, h->buf0, h->buf1, g.ix * g.iy, g.iz, g.bz, g.ix, g.iz * g.ix, 1, g.ix,
                        "Z")))
            return rc;
    }
    mark(2);
    heat_y_fold_kernel<<<dim3((g.ix + 127) / 128, 2, g.iz), b1, 0, st>>>(theta, h->buf1, g);
    CK(cudaGetLastError());
    mark(3);
    if (tile_plan(g.iy, false, 8, 1, true, true).sys != 0) {
        // Y sweep: system kk * ix + ii, row jj; the solution goes straight into
        // the X sweep's layout [ii][kk][jj] (rows contiguous: staged and stored
        // coalesced), then the X wall folds on its two wall planes
        if ((rc = sweep(1, h->buf1, h->buf0, g.ix * g.iz, g.iy, g.by, g.ix, g.iy, g.iz * g.iy, 1,
                        "Y")))
            return rc;
        mark(4);
        heat_x_fold_kernel<<<dim3((g.iy + 127) / 128, 2, g.iz), b1, 0, st>>>(theta, h->buf0, g);
    } else {
        if ((rc = sweep(1, h->buf1, h->buf1, g.ix * g.iz, g.iy, g.by, 0, 0, 0, 0, "Y")))
            return rc;
        mark(4);
        heat_y_to_x_kernel<<<dim3(tx, ty, g.iz), bt, 0, st>>>(theta, h->buf1, h->buf0, g);
    }
    CK(cudaGetLastError());
    mark(5);
    // X sweep: system kk * iy + jj, row ii; the solution goes straight into
    // theta's interior (update_theta_kernel's copy, solve_theta.cu:335-347):
    // a system's rows are contiguous there, so the sweep stages them in shared
    // memory and stores them coalesced
    const int plane = (g.ix + 2) * (g.iy + 2);
    if ((rc = sweep(2, h->buf0, theta + plane + (g.ix + 2) + 1, g.iy * g.iz, g.ix, g.bx, g.iy,
                    plane, g.ix + 2, 1, "X")))
        return rc;
    mark(6);
    mark(7);
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
    {
        const double bx = dt / (2.0 * (2.0 / ix) * (2.0 / ix));
        const double by = dt / (2.0 * (2.0 / iy) * (2.0 / iy));
        CKH(upload(&h->hpar, {bx, by, dt * 3.0 * HEAT_PI * HEAT_PI, (double)iy, (double)iz}));
    }
    const size_t inner = (size_t)ix * iy * iz;
    CKH(cudaMalloc(&h->buf0, sizeof(double) * inner));
    CKH(cudaMalloc(&h->buf1, sizeof(double) * inner));
    CKH(cudaMalloc(&h->err, sizeof(double)));
    CKH(cudaMalloc(&h->scratch, sizeof(double) * (size_t)(ix + 2) * (iy + 2) * (iz + 2)));
    h->tab_stride = gen_table_doubles(std::max(ix, std::max(iy, iz)));
    CKH(cudaMalloc(&h->tab, sizeof(double) * 3 * h->tab_stride));
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
    // the factor tables of the three sweeps, once: each direction's matrix is
    // fixed by the grid and dt (fully implicit walls, cbound)
    const int rows[3] = {iz, iy, ix};
    const double base[3] = {g.bz, g.by, g.bx};
    for (int d = 0; d < 3; ++d) {
        TileArgs ga = {};
        ga.cs = base[d];
        ga.cbound = 1;
        const int rc = build_gen_table<1>(rows[d], ga, h->tab + d * h->tab_stride, h->cap);
        if (rc) return cleanup(rc);
    }
    const cudaError_t e = cudaStreamSynchronize(h->cap);
    if (e != cudaSuccess)
        return cleanup(fail(BTDMA_ERR_CUDA, "heat factor tables: %s", cudaGetErrorString(e)));
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
    cudaFree(h->hpar);
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
    cudaEvent_t ev[8] = {};
    for (auto& e : ev) CK(cudaEventCreate(&e));
    int rc = heat_enqueue(h, theta, stream, ev);
    if (!rc && cudaEventSynchronize(ev[7]) != cudaSuccess)
        rc = fail(BTDMA_ERR_CUDA, "profiled heat step failed");
    if (!rc) {
        auto sec = [&](int a, int b) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[a], ev[b]);
            return 1e-3 * ms;
        };
        // the reference's 12 events (solve_theta.cu:436-439): rhs, solve_z,
        // solve_y, solve_x, etc, comm, tdma_{z,y,x}_comm, tdma_{z,y,x}_gpu
        const double t[12] = {sec(0, 1), sec(1, 3), sec(3, 5), sec(5, 7), 0.0,       0.0,
                              0.0,       0.0,       0.0,       sec(1, 2), sec(3, 4), sec(5, 6)};
        std::memcpy(times, t, sizeof t);
        h->last_stream = stream;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
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
    double* buf = nullptr;   // nx * ny * nz, the sweep layout
    double* buf2 = nullptr;  // a second one: the fused step's y-sweep input
    // factor tables per (dir, comp), gstride apart, and what each was last
    // built for: reused while the coefficient and the stream stay the same.
    // A second set of 9 tables serves captured sweeps: a graph rebuilds its
    // tables on every replay, and must not overwrite the cached ones (a later
    // uncaptured call with the cached key would then use the graph's tables).
    double* gtab = nullptr;
    size_t gstride = 0;
    struct TabKey {
        bool valid = false;
        double c = 0.0;
        cudaStream_t stream = nullptr;
    } gkey[3][3];
    unsigned* status = nullptr;
    // Array-based backend (btdma_momentum_set_backend): the method and
    // segments of the per-direction library handles, the raw axis factors
    // [dir][comp][ar, cr][n] and the explicit A, B, C, X of a sweep.
    int backend = BTDMA_PASCAL;
    double eps_constant = 1.0e-12;
    double* raw = nullptr;
    size_t raw_off[3][3] = {};
    double* coef = nullptr;  // A, B, C, X, each nx * ny * nz
    btdma_t hd[3] = {};
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
    if ((long long)(nx + 2) * (ny + 2) * (nz + 2) >= (1LL << 31))
        return fail(BTDMA_ERR_SIZE, "ghosted grid above 2^31 cells");
    // row tables (MomentumSolverGPU.cu:135-155, :176-180, :205-209): for row
    // r = 1..n, staggered when comp == dir;  a = -c ta, c = -c tc, b = 1 + c tb
    const double* dxs[3] = {dx0, dx1, dx2};
    const double* dms[3] = {dmx0, dmx1, dmx2};
    std::vector<double> tab, raw;
    size_t off[3][3], roff[3][3];
    for (int d = 0; d < 3; ++d)
        for (int comp = 0; comp < 3; ++comp) {
            off[d][comp] = tab.size();
            roff[d][comp] = raw.size();
            const int m = n[d];
            std::vector<double> ta(m), tb(m), tc(m), ra(m), rc(m);
            const double* dx = dxs[d];
            const double* dm = dms[d];
            for (int r = 1; r <= m; ++r) {
                const double ar = comp == d ? 1.0 / (dm[r] * dx[r - 1]) : 1.0 / (dx[r] * dm[r]);
                const double cr = comp == d ? 1.0 / (dm[r] * dx[r]) : 1.0 / (dx[r] * dm[r + 1]);
                ra[r - 1] = ar;
                rc[r - 1] = cr;
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
            raw.insert(raw.end(), ra.begin(), ra.end());
            raw.insert(raw.end(), rc.begin(), rc.end());
        }
    btdma_momentum* h = new btdma_momentum();
    h->g.nx = nx;
    h->g.ny = ny;
    h->g.nz = nz;
    h->pbc[0] = pbc_x ? 1 : 0;
    h->pbc[1] = pbc_y ? 1 : 0;
    std::memcpy(h->tab_off, off, sizeof off);
    std::memcpy(h->raw_off, roff, sizeof roff);
    h->gstride = gen_table_doubles(std::max(nx, std::max(ny, nz)));
    auto cleanup = [&](int code) {
        btdma_momentum_destroy(h);
        return code;
    };
    if (cudaMalloc(&h->tab, sizeof(double) * tab.size()) != cudaSuccess ||
        cudaMemcpy(h->tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMalloc(&h->buf, sizeof(double) * (size_t)nx * ny * nz) != cudaSuccess ||
        cudaMalloc(&h->buf2, sizeof(double) * (size_t)nx * ny * nz) != cudaSuccess ||
        cudaMalloc(&h->gtab, sizeof(double) * 18 * h->gstride) != cudaSuccess ||
        cudaMalloc(&h->raw, sizeof(double) * raw.size()) != cudaSuccess ||
        cudaMemcpy(h->raw, raw.data(), sizeof(double) * raw.size(), cudaMemcpyHostToDevice) !=
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
    cudaFree(h->buf2);
    cudaFree(h->gtab);
    cudaFree(h->status);
    cudaFree(h->raw);
    cudaFree(h->coef);
    for (auto& d : h->hd) btdma_destroy(d);
    delete h;
    return BTDMA_OK;
}

int btdma_momentum_set_backend(btdma_momentum_t h, int method, int P, int flags,
                               double eps_constant) {
    if (!h) return fail(BTDMA_ERR_ARG, "null handle");
    if (method < BTDMA_PASCAL || method > BTDMA_FILTERED_V2)
        return fail(BTDMA_ERR_ARG, "unknown method %d", method);
    if (method != BTDMA_PASCAL && P < 1) return fail(BTDMA_ERR_ARG, "P must be >= 1");
    if (!(eps_constant > 0.0)) return fail(BTDMA_ERR_ARG, "eps_constant must be positive");
    for (auto& d : h->hd) {
        btdma_destroy(d);
        d = nullptr;
    }
    h->backend = BTDMA_PASCAL;
    if (method == BTDMA_PASCAL) return BTDMA_OK;
    const MomGeom& g = h->g;
    const int n[3] = {g.nx, g.ny, g.nz};
    const size_t cells = (size_t)g.nx * g.ny * g.nz;
    if (!h->coef && cudaMalloc(&h->coef, sizeof(double) * 4 * cells) != cudaSuccess)
        return fail(BTDMA_ERR_CUDA, "momentum coefficient arrays: %s",
                    cudaGetErrorString(cudaGetLastError()));
    for (int d = 0; d < 3; ++d) {
        const int rc = btdma_create(method, (int)(cells / n[d]), n[d], P, BTDMA_FP64, flags,
                                    &h->hd[d]);
        if (rc) {
            for (auto& x : h->hd) {
                btdma_destroy(x);
                x = nullptr;
            }
            return rc;
        }
        btdma_set_eps_constant(h->hd[d], eps_constant);
    }
    h->backend = method;
    h->eps_constant = eps_constant;
    return BTDMA_OK;
}

namespace {

// One momentum sweep of the tiled solve with generated coefficients: D in the
// sweep's layout (system index fastest), or for the z sweep (zfield non-null)
// the ghosted field itself, read by the sweep without a gather (pin: the w
// component's row 0 is x = 0); x stored through the layout map (system s, row
// r -> X + (s / xblk) xbs + (s % xblk) xss + r xrs).  Returns 0 with `taken`
// false when a zfield sweep's shape is not tiled that way.  This
// (dir, comp)'s factor table is built here unless the last build was for the
// same coefficient on the same stream; inside a stream capture it is always
// built, into the capture set of tables, so that a graph carries its own
// tables and its replays leave the cached ones intact.
int mom_tile_sweep(btdma_momentum_t h, int dir, int comp, const double* D, double* X, int xblk,
                   int xbs, int xss, int xrs, double c, cudaStream_t stream,
                   const double* zfield = nullptr, bool* taken = nullptr) {
    const MomGeom& g = h->g;
    const int n[3] = {g.nx, g.ny, g.nz};
    const int n_sys = g.nx * g.ny * g.nz / n[dir];
    TileArgs t = {};
    t.cs = c;
    t.ga = h->tab + h->tab_off[dir][comp];
    t.gb = t.ga + n[dir];
    t.gc = t.gb + n[dir];
    t.xblk = xblk;
    t.xbs = xbs;
    t.xss = xss;
    t.xrs = xrs;
    auto& key = h->gkey[dir][comp];
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(stream, &cap));
    const bool capturing = cap != cudaStreamCaptureStatusNone;
    const bool ready = !capturing && key.valid && key.c == c && key.stream == stream;
    double* const gt =
        h->gtab + (size_t)((capturing ? 9 : 0) + dir * 3 + comp) * h->gstride;
    if (!ready && !capturing) key.valid = false;  // rebuilt below
    const bool cyc = dir < 2 && h->pbc[dir] != 0;
    int rc;
    if (zfield) {
        rc = try_mom_z(zfield, X, g.nx, g.ny, g.nz, t, comp == 2 ? 1 : 0, h->status, stream, gt,
                       ready);
        if (taken) *taken = rc == 1;
        if (rc == 0) return BTDMA_OK;  // the caller gathers instead
    } else {
        rc = cyc ? try_tile_gen<3, true>(D, X, n_sys, n[dir], t, h->status, stream, gt, ready)
                 : try_tile_gen<3, false>(D, X, n_sys, n[dir], t, h->status, stream, gt, ready);
    }
    if (rc != 1) return rc < 0 ? rc : fail(BTDMA_ERR_UNSUPPORTED, "sweep not tileable");
    if (!capturing) {
        key.valid = true;
        key.c = c;
        key.stream = stream;
    }
    return BTDMA_OK;
}

}  // namespace

int btdma_momentum_sweep(btdma_momentum_t h, int dir, int comp, const double* q, double* dst,
                         double c, cudaStream_t stream) {
    if (!h || !q || !dst) return fail(BTDMA_ERR_ARG, "null argument");
    if (dir < 0 || dir > 2 || comp < 0 || comp > 2)
        return fail(BTDMA_ERR_ARG, "dir and comp must be 0, 1 or 2");
    const MomGeom& g = h->g;
    const int n[3] = {g.nx, g.ny, g.nz};
    const int n_sys = g.nx * g.ny * g.nz / n[dir];
    if (h->backend != BTDMA_PASCAL) {
        // the reference's sequence (adi_{z,y,x}_): build A, B, C, D, set rho
        // from system 0's column, solve with the handle's method, scatter
        const size_t cells = (size_t)g.nx * g.ny * g.nz;
        double* A = h->coef;
        double* B = A + cells;
        double* C = B + cells;
        double* X = C + cells;
        const dim3 b1(128, 1, 1), bt(MOM_TILE, 8, 1);
        if (dir == 2)
            mom_gather_kernel<2><<<dim3((g.nx + 127) / 128, (g.ny + MOM_GR - 1) / MOM_GR, g.nz),
                                   b1, 0, stream>>>(q, h->buf, g, comp == 2 ? 1 : 0);
        else if (dir == 1)
            mom_gather_kernel<1><<<dim3((g.nx + 127) / 128, (g.nz + MOM_GR - 1) / MOM_GR, g.ny),
                                   b1, 0, stream>>>(q, h->buf, g, 0);
        else
            mom_gather_x_kernel<<<dim3((g.nx + MOM_TILE - 1) / MOM_TILE,
                                       (g.ny + MOM_TILE - 1) / MOM_TILE, g.nz), bt, 0, stream>>>(
                q, h->buf, g);
        CK(cudaGetLastError());
        const double* ra = h->raw + h->raw_off[dir][comp];
        mom_coef_kernel<<<std::min<size_t>((cells + 255) / 256, 148 * 16), 256, 0, stream>>>(
            A, B, C, ra, ra + n[dir], n[dir], n_sys, c, dir == 2 ? 1 : 0, comp == 2 ? 1 : 0);
        CK(cudaGetLastError());
        const bool cyc = dir < 2 && h->pbc[dir] != 0;
        btdma_t hd = h->hd[dir];
        int rc = btdma_set_rho(hd, A, B, C, n_sys, n[dir], stream);
        if (!rc) rc = btdma_solve_out(hd, A, B, C, h->buf, X, n_sys, n[dir], cyc ? 1 : 0, stream);
        if (rc) return rc;
        if (dir == 2)
            mom_scatter_kernel<2><<<dim3((g.nx + 127) / 128, (g.ny + MOM_GR - 1) / MOM_GR, g.nz),
                                    b1, 0, stream>>>(X, dst, g);
        else if (dir == 1)
            mom_scatter_kernel<1><<<dim3((g.nx + 127) / 128, (g.nz + MOM_GR - 1) / MOM_GR, g.ny),
                                    b1, 0, stream>>>(X, dst, g);
        else
            mom_scatter_x_kernel<<<dim3((g.ny + MOM_TILE - 1) / MOM_TILE,
                                        (g.nx + MOM_TILE - 1) / MOM_TILE, g.nz), bt, 0, stream>>>(
                X, dst, g);
        CK(cudaGetLastError());
        return BTDMA_OK;
    }
    const dim3 b1(128, 1, 1), bt(MOM_TILE, 8, 1);
    const int sp = (g.nx + 2) * (g.ny + 2);  // plane stride (< 2^31, checked at create)
    double* const dst_in = dst + sp + (g.nx + 2) + 1;  // dst(1, 1, 1)
    if (dir == 2) {
        // z: system s = (j, i), i = s % nx fastest, row r -> dst(i, j, k = r + 1);
        // read from q directly unless q is dst (in place: other CTAs' stores
        // would land in rows still to be read) or the shape is not tiled so
        bool taken = false;
        if (q != dst) {
            const int rc = mom_tile_sweep(h, 2, comp, nullptr, dst_in, g.nx, g.nx + 2, 1, sp, c,
                                          stream, q, &taken);
            if (rc || taken) return rc;
        }
        mom_gather_kernel<2><<<dim3((g.nx + 127) / 128, (g.ny + MOM_GR - 1) / MOM_GR, g.nz), b1,
                                 0, stream>>>(q, h->buf, g, comp == 2 ? 1 : 0);
        CK(cudaGetLastError());
        return mom_tile_sweep(h, 2, comp, h->buf, dst_in, g.nx, g.nx + 2, 1, sp, c, stream);
    }
    if (dir == 1) {
        // y: system s = (k, i), row r -> dst(i, j = r + 1, k)
        mom_gather_kernel<1><<<dim3((g.nx + 127) / 128, (g.nz + MOM_GR - 1) / MOM_GR, g.ny), b1,
                                 0, stream>>>(q, h->buf, g, 0);
        CK(cudaGetLastError());
        return mom_tile_sweep(h, 1, comp, h->buf, dst_in, g.nx, sp, 1, g.nx + 2, c, stream);
    }
    // x: system s = (k, j), j = s % ny fastest, row r -> dst(i = r + 1, j, k): a
    // system's rows are contiguous in the field, so the sweep stages them and
    // stores them coalesced (no transposing scatter)
    mom_gather_x_kernel<<<dim3((g.nx + MOM_TILE - 1) / MOM_TILE, (g.ny + MOM_TILE - 1) / MOM_TILE,
                               g.nz), bt, 0, stream>>>(q, h->buf, g);
    CK(cudaGetLastError());
    return mom_tile_sweep(h, 0, comp, h->buf, dst_in, g.ny, sp, g.nx + 2, 1, c, stream);
}

int btdma_momentum_adi(btdma_momentum_t h, int comp, double* rhs, double* q_out, double c,
                       cudaStream_t stream) {
    if (!h || !rhs || !q_out) return fail(BTDMA_ERR_ARG, "null argument");
    if (comp < 0 || comp > 2) return fail(BTDMA_ERR_ARG, "comp must be 0, 1 or 2");
    if (h->backend != BTDMA_PASCAL) {  // the reference's sequence, z and y in place on rhs
        int rc = btdma_momentum_sweep(h, 2, comp, rhs, rhs, c, stream);
        if (!rc) rc = btdma_momentum_sweep(h, 1, comp, rhs, rhs, c, stream);
        if (!rc) rc = btdma_momentum_sweep(h, 0, comp, rhs, q_out, c, stream);
        return rc;
    }
    // Each sweep stores its solution straight into the next sweep's layout:
    // z (read from rhs itself) -> y layout [j][k][i] (mapped rows), y -> x
    // layout [i][k][j] (contiguous rows: staged, coalesced), x -> q_out's
    // interior (staged); rhs is only read.
    const MomGeom& g = h->g;
    const dim3 b1(128, 1, 1);
    const int sp = (g.nx + 2) * (g.ny + 2);
    bool taken = false;  // the z sweep reads rhs directly when its shape allows
    int rc = mom_tile_sweep(h, 2, comp, nullptr, h->buf2, g.nx, g.nx * g.nz, 1, g.nx, c, stream,
                            rhs, &taken);
    if (!rc && !taken) {
        mom_gather_kernel<2><<<dim3((g.nx + 127) / 128, (g.ny + MOM_GR - 1) / MOM_GR, g.nz), b1,
                               0, stream>>>(rhs, h->buf, g, comp == 2 ? 1 : 0);
        CK(cudaGetLastError());
        rc = mom_tile_sweep(h, 2, comp, h->buf, h->buf2, g.nx, g.nx * g.nz, 1, g.nx, c, stream);
    }
    if (!rc)
        rc = mom_tile_sweep(h, 1, comp, h->buf2, h->buf, g.nx, g.ny, g.nz * g.ny, 1, c, stream);
    if (!rc)
        rc = mom_tile_sweep(h, 0, comp, h->buf, q_out + sp + (g.nx + 2) + 1, g.ny, sp, g.nx + 2,
                            1, c, stream);
    return rc;
}

int btdma_momentum_status(btdma_momentum_t h, unsigned* status, cudaStream_t stream) {
    if (!h || !status) return fail(BTDMA_ERR_ARG, "null argument");
    CK(cudaMemcpyAsync(status, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    CK(cudaMemsetAsync(h->status, 0, sizeof(unsigned), stream));
    CK(cudaStreamSynchronize(stream));
    for (btdma_t hd : h->hd) {  // the array-based backend's handles
        if (!hd) continue;
        unsigned s = 0;
        const int rc = btdma_status(hd, &s);
        if (rc) return rc;
        *status |= s;
    }
    return BTDMA_OK;
}
