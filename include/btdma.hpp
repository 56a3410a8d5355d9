// Header-only C++ drop-in for the reference's CUDA solver classes, on top of the
// C ABI in btdma.h (link with libbtdma.so).
//
//   PaScaLTDMACUDA    libs/pascal_tdma/include/pascal_tdma_cuda.hpp:18-56
//   FilteredTDMACUDA  libs/filtered_tdma/include/filtered_tdma_cuda.hpp:161-266
//   TdmaBackendGPU    apps/heat_gpu/tdma_backend_gpu.hpp:21-70
//
// Same class names, constructor argument order and method names.  Differences:
//   * `nprocs` is the number of segments P each system is split into inside the
//     GPU (there are no ranks); `myrank`, `comm`, `left_rank`, `right_rank`,
//     `block_x`, `block_y` are accepted and ignored.  The communicator type is a
//     template parameter, so the header compiles with or without <mpi.h>.
//   * arrays hold the whole system ([n_row x n_sys], all P segments), not one
//     rank's slab.
//   * A, B and C are left unchanged; D <- x.
//   * errors throw btdma::Error (the reference aborts the process).
//   * last_comm_ms() is always 0; last_gpu_ms() is the CUDA-event time of the
//     last *_profile call, as in the reference.
//   * solves run on the stream given by set_stream() (default: the legacy
//     default stream, as the reference).
#pragma once

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cctype>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "btdma.h"

namespace btdma {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != BTDMA_OK) throw Error(rc, std::string("btdma: ") + btdma_last_error());
}

// Owning handle.
class Handle {
   public:
    Handle(int method, int n_sys, int n_row, int P, int precision = BTDMA_FP64, int flags = 0) {
        check(btdma_create(method, n_sys, n_row, P, precision, flags, &h_));
        n_sys_ = n_sys;
        n_row_ = n_row;
    }
    ~Handle() { btdma_destroy(h_); }
    Handle(const Handle&) = delete;
    Handle& operator=(const Handle&) = delete;
    btdma_t get() const { return h_; }
    int n_sys() const { return n_sys_; }
    int n_row() const { return n_row_; }

   private:
    btdma_t h_ = nullptr;
    int n_sys_ = 0, n_row_ = 0;
};

// CUDA-event timing of one call (last_gpu_ms of the *_profile variants).
class EventTimer {
   public:
    EventTimer() {
        cudaEventCreate(&e0_);
        cudaEventCreate(&e1_);
    }
    ~EventTimer() {
        cudaEventDestroy(e0_);
        cudaEventDestroy(e1_);
    }
    template <class F>
    double time(cudaStream_t st, F&& f) {
        cudaEventRecord(e0_, st);
        f();
        cudaEventRecord(e1_, st);
        cudaEventSynchronize(e1_);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0_, e1_);
        return ms;
    }

   private:
    cudaEvent_t e0_ = nullptr, e1_ = nullptr;
};

}  // namespace btdma

class PaScaLTDMACUDA {
   public:
    template <class Comm = int>
    PaScaLTDMACUDA(int n_sys, int myrank, int nprocs, Comm comm = Comm(), int block_x = 128,
                   int block_y = 1)
        : n_sys_(n_sys), nprocs_(nprocs) {
        (void)myrank;
        (void)comm;
        (void)block_x;
        (void)block_y;
    }
    PaScaLTDMACUDA(const PaScaLTDMACUDA&) = delete;
    PaScaLTDMACUDA& operator=(const PaScaLTDMACUDA&) = delete;

    void solve(double* d_A, double* d_B, double* d_C, double* d_D, int n_sys, int n_row) {
        btdma::check(btdma_solve(get(n_sys, n_row), d_A, d_B, d_C, d_D, n_sys, n_row, stream_));
    }
    void solve_cyclic(double* d_A, double* d_B, double* d_C, double* d_D, int n_sys, int n_row) {
        btdma::check(
            btdma_solve_cyclic(get(n_sys, n_row), d_A, d_B, d_C, d_D, n_sys, n_row, stream_));
    }
    void solve_profile(double* d_A, double* d_B, double* d_C, double* d_D, int n_sys, int n_row) {
        gpu_ms_ = timer_.time(stream_, [&] { solve(d_A, d_B, d_C, d_D, n_sys, n_row); });
    }
    void solve_cyclic_profile(double* d_A, double* d_B, double* d_C, double* d_D, int n_sys,
                              int n_row) {
        gpu_ms_ = timer_.time(stream_, [&] { solve_cyclic(d_A, d_B, d_C, d_D, n_sys, n_row); });
    }

    int n_sys_rt() const { return n_sys_; }
    int n_row_rt() const { return 2 * nprocs_; }
    int nprocs() const { return nprocs_; }
    double last_comm_ms() const { return 0.0; }
    double last_gpu_ms() const { return gpu_ms_; }
    void set_stream(cudaStream_t s) { stream_ = s; }
    // BTDMA_TILE_AUTO / NARROW / WIDE (btdma_set_tile_shape); kept across handle regrowth.
    void set_tile_shape(int shape) {
        tile_shape_ = shape;
        if (h_) btdma::check(btdma_set_tile_shape(h_->get(), shape));
    }

   private:
    // The handle is sized on the first solve (n_row is not a constructor
    // argument of the reference class) and grown only if a later solve needs it.
    btdma_t get(int n_sys, int n_row) {
        if (!h_ || n_row > h_->n_row() || n_sys > h_->n_sys()) {
            h_.reset();
            h_.reset(new btdma::Handle(BTDMA_PASCAL, std::max(n_sys, n_sys_), n_row, nprocs_));
            btdma::check(btdma_set_tile_shape(h_->get(), tile_shape_));
        }
        return h_->get();
    }
    int tile_shape_ = BTDMA_TILE_AUTO;
    int n_sys_, nprocs_;
    std::unique_ptr<btdma::Handle> h_;
    cudaStream_t stream_ = 0;
    btdma::EventTimer timer_;
    double gpu_ms_ = 0.0;
};

class FilteredTDMACUDA {
   public:
    template <class Comm = int>
    FilteredTDMACUDA(int n_sys, int n_row, int myrank, int nprocs, Comm comm = Comm(),
                     int left_rank = -2, int right_rank = -2, double eps_constant = 1.0e-12,
                     int flags = 0)
        : n_sys_(n_sys), n_row_(n_row), nprocs_(nprocs),
          h_(BTDMA_FILTERED_V2, n_sys, n_row, nprocs, BTDMA_FP64, flags) {
        (void)myrank;
        (void)comm;
        (void)left_rank;
        (void)right_rank;
        btdma::check(btdma_set_eps_constant(h_.get(), eps_constant));
    }
    FilteredTDMACUDA(const FilteredTDMACUDA&) = delete;
    FilteredTDMACUDA& operator=(const FilteredTDMACUDA&) = delete;

    void solve_filtered_v1(double* A, double* B, double* C, double* D) { run(BTDMA_FILTERED_V1, A, B, C, D, false); }
    void solve_filtered_v2(double* A, double* B, double* C, double* D) { run(BTDMA_FILTERED_V2, A, B, C, D, false); }
    void solve_cycl_filtered_v1(double* A, double* B, double* C, double* D) { run(BTDMA_FILTERED_V1, A, B, C, D, true); }
    void solve_cycl_filtered_v2(double* A, double* B, double* C, double* D) { run(BTDMA_FILTERED_V2, A, B, C, D, true); }

    void solve_filtered_v1_profile(double* A, double* B, double* C, double* D) {
        gpu_ms_ = timer_.time(stream_, [&] { solve_filtered_v1(A, B, C, D); });
    }
    void solve_filtered_v2_profile(double* A, double* B, double* C, double* D) {
        gpu_ms_ = timer_.time(stream_, [&] { solve_filtered_v2(A, B, C, D); });
    }
    void solve_cycl_filtered_v1_profile(double* A, double* B, double* C, double* D) {
        gpu_ms_ = timer_.time(stream_, [&] { solve_cycl_filtered_v1(A, B, C, D); });
    }
    void solve_cycl_filtered_v2_profile(double* A, double* B, double* C, double* D) {
        gpu_ms_ = timer_.time(stream_, [&] { solve_cycl_filtered_v2(A, B, C, D); });
    }

    void set_rho_device(const double* d_A, const double* d_B, const double* d_C) {
        btdma::check(btdma_set_rho(h_.get(), d_A, d_B, d_C, n_sys_, n_row_, stream_));
    }
    void set_eps_constant(double eps_constant) {
        btdma::check(btdma_set_eps_constant(h_.get(), eps_constant));
    }
    // J of the first segment (the reference reports its own rank's J).
    int last_J() const {
        int J = -1, n = 0;
        btdma::check(btdma_last_J(h_.get(), &J, 1, &n));
        return J;
    }

    int n_sys() const { return n_sys_; }
    int n_row() const { return n_row_; }
    int nprocs() const { return nprocs_; }
    double last_comm_ms() const { return 0.0; }
    double last_gpu_ms() const { return gpu_ms_; }
    void set_stream(cudaStream_t s) { stream_ = s; }

   private:
    void run(int method, double* A, double* B, double* C, double* D, bool cyclic) {
        btdma::check(btdma_set_method(h_.get(), method));
        if (cyclic)
            btdma::check(btdma_solve_cyclic(h_.get(), A, B, C, D, n_sys_, n_row_, stream_));
        else
            btdma::check(btdma_solve(h_.get(), A, B, C, D, n_sys_, n_row_, stream_));
    }
    int n_sys_, n_row_, nprocs_;
    btdma::Handle h_;
    cudaStream_t stream_ = 0;
    btdma::EventTimer timer_;
    double gpu_ms_ = 0.0;
};

class TdmaBackendGPU {
   public:
    enum class Kind { FILTERED, FILTERED_V2, PASCAL };

    // Case-insensitive: "pascal" | "pascal_tdma" -> PASCAL, "filtered_v2" ->
    // FILTERED_V2, anything else -> FILTERED (apps/heat_gpu/tdma_backend_gpu.cu:6-13).
    static Kind parse(const std::string& s) {
        std::string t;
        for (char c : s) t.push_back(static_cast<char>(std::tolower(static_cast<unsigned char>(c))));
        if (t == "pascal" || t == "pascal_tdma") return Kind::PASCAL;
        if (t == "filtered_v2") return Kind::FILTERED_V2;
        return Kind::FILTERED;
    }

    template <class Comm = int>
    TdmaBackendGPU(Kind kind, int n_sys, int n_row, int myrank, int nprocs, Comm comm,
                   int left_rank, int right_rank, double eps_constant)
        : kind_(kind), n_sys_(n_sys), n_row_(n_row) {
        if (kind_ == Kind::PASCAL)
            pasc_.reset(new PaScaLTDMACUDA(n_sys, myrank, nprocs, comm, 128, 1));
        else
            filt_.reset(new FilteredTDMACUDA(n_sys, n_row, myrank, nprocs, comm, left_rank,
                                             right_rank, eps_constant));
    }

    // The heat app routes every backend through its profile variant
    // (apps/heat_gpu/tdma_backend_gpu.cu:35-46); so does this class.
    void solve(double* d_A, double* d_B, double* d_C, double* d_D) {
        if (kind_ == Kind::FILTERED)
            filt_->solve_filtered_v1_profile(d_A, d_B, d_C, d_D);
        else if (kind_ == Kind::FILTERED_V2)
            filt_->solve_filtered_v2_profile(d_A, d_B, d_C, d_D);
        else
            pasc_->solve_profile(d_A, d_B, d_C, d_D, n_sys_, n_row_);
    }
    void solve_cyclic(double* d_A, double* d_B, double* d_C, double* d_D) {
        if (kind_ == Kind::FILTERED)
            filt_->solve_cycl_filtered_v1_profile(d_A, d_B, d_C, d_D);
        else if (kind_ == Kind::FILTERED_V2)
            filt_->solve_cycl_filtered_v2_profile(d_A, d_B, d_C, d_D);
        else
            pasc_->solve_cyclic_profile(d_A, d_B, d_C, d_D, n_sys_, n_row_);
    }
    void set_rho_device(const double* d_A, const double* d_B, const double* d_C) {
        if (kind_ != Kind::PASCAL) filt_->set_rho_device(d_A, d_B, d_C);
    }
    void set_eps_constant(double eps_constant) {
        if (kind_ != Kind::PASCAL) filt_->set_eps_constant(eps_constant);
    }
    Kind kind() const { return kind_; }
    double last_comm_ms() const { return 0.0; }
    double last_gpu_ms() const {
        return kind_ == Kind::PASCAL ? pasc_->last_gpu_ms() : filt_->last_gpu_ms();
    }
    void set_stream(cudaStream_t s) {
        if (pasc_) pasc_->set_stream(s);
        if (filt_) filt_->set_stream(s);
    }

   private:
    Kind kind_;
    int n_sys_, n_row_;
    std::unique_ptr<FilteredTDMACUDA> filt_;
    std::unique_ptr<PaScaLTDMACUDA> pasc_;
};

// ------------------------------------------------------------------------
// RAII wrappers of the components with no reference class of their own
// (ragged batches, the fused heat step, the channel Poisson and momentum
// sweeps); each owns one C-ABI handle and throws btdma::Error on failure.
namespace btdma {

class HeatADI {
   public:
    HeatADI(int ix, int iy, int iz, double dt) { check(btdma_heat_create(ix, iy, iz, dt, &h_)); }
    ~HeatADI() { btdma_heat_destroy(h_); }
    HeatADI(const HeatADI&) = delete;
    HeatADI& operator=(const HeatADI&) = delete;
    void init(double* d_theta, cudaStream_t s = 0) { check(btdma_heat_init(h_, d_theta, s)); }
    void step(double* d_theta, int n_steps, bool graph = true, cudaStream_t s = 0) {
        check(btdma_heat_step(h_, d_theta, n_steps, graph ? 1 : 0, s));
    }
    double l2_error(const double* d_theta, double t_phys) {
        double l2 = 0.0;
        check(btdma_heat_l2_error(h_, d_theta, t_phys, &l2));
        return l2;
    }

   private:
    btdma_heat_t h_ = nullptr;
};

class ChannelPoisson {
   public:
    ChannelPoisson(int nz, const double* dz, const double* dmz, int n_modes, const double* lambda,
                   bool pin_mode0 = true) {
        check(btdma_poisson_create(nz, dz, dmz, n_modes, lambda, pin_mode0 ? 1 : 0, &h_));
    }
    ~ChannelPoisson() { btdma_poisson_destroy(h_); }
    ChannelPoisson(const ChannelPoisson&) = delete;
    ChannelPoisson& operator=(const ChannelPoisson&) = delete;
    // d_hat: complex [nz][n_modes] as interleaved doubles, in place
    void solve(double* d_hat, cudaStream_t s = 0) { check(btdma_poisson_solve(h_, d_hat, s)); }

   private:
    btdma_poisson_t h_ = nullptr;
};

class ChannelMomentum {
   public:
    ChannelMomentum(int nx, int ny, int nz, const double* dx0, const double* dmx0,
                    const double* dx1, const double* dmx1, const double* dx2, const double* dmx2,
                    bool pbc_x, bool pbc_y) {
        check(btdma_momentum_create(nx, ny, nz, dx0, dmx0, dx1, dmx1, dx2, dmx2, pbc_x ? 1 : 0,
                                    pbc_y ? 1 : 0, &h_));
    }
    ~ChannelMomentum() { btdma_momentum_destroy(h_); }
    ChannelMomentum(const ChannelMomentum&) = delete;
    ChannelMomentum& operator=(const ChannelMomentum&) = delete;
    void adi(int comp, double* d_rhs, double* d_q, double nu_dt_half, cudaStream_t s = 0) {
        check(btdma_momentum_adi(h_, comp, d_rhs, d_q, nu_dt_half, s));
    }

   private:
    btdma_momentum_t h_ = nullptr;
};

// Ragged (CSR) batches through a PaScaL handle of the given storage precision.
class RaggedSolver {
   public:
    explicit RaggedSolver(int n_sys, int precision = BTDMA_FP64) {
        check(btdma_create(BTDMA_PASCAL, n_sys, 64, 2, precision, 0, &h_));
    }
    ~RaggedSolver() { btdma_destroy(h_); }
    RaggedSolver(const RaggedSolver&) = delete;
    RaggedSolver& operator=(const RaggedSolver&) = delete;
    void solve(const double* A, const double* B, const double* C, const double* D, double* X,
               const long long* row_offsets, const unsigned char* periodic, int n_sys,
               cudaStream_t s = 0) {
        check(btdma_solve_ragged(h_, A, B, C, D, X, row_offsets, periodic, n_sys, s));
    }
    void autotune(const double* A, const double* B, const double* C, const double* D, double* X,
                  const long long* row_offsets, const unsigned char* periodic, int n_sys,
                  cudaStream_t s = 0) {
        check(btdma_ragged_autotune(h_, A, B, C, D, X, row_offsets, periodic, n_sys, s));
    }
    // The current plan (e.g. after autotune), and a stored plan applied again
    // to the same layout without timing.
    std::vector<btdma_ragged_bucket> plan() const {
        int n = 0;
        check(btdma_ragged_plan_info(h_, nullptr, 0, &n));
        std::vector<btdma_ragged_bucket> out(n);
        check(btdma_ragged_plan_info(h_, out.data(), n, &n));
        return out;
    }
    void set_plan(const std::vector<btdma_ragged_bucket>& plan) {
        check(btdma_ragged_set_plan(h_, plan.data(), (int)plan.size()));
    }

   private:
    btdma_t h_ = nullptr;
};

}  // namespace btdma
