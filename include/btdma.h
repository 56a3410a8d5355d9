/*
 * btdma — batched tridiagonal solves on one NVIDIA B200 (sm_100a).
 *
 * C ABI of the library.  Every array is a caller-owned DEVICE pointer (except
 * the host arrays of btdma_solve_host) in the
 * reference's row-interleaved layout [n_row x n_sys]: row j of system i at
 * j*n_sys + i (reference: libs/pascal_tdma/include/pascal_tdma.hpp:13,
 * libs/filtered_tdma/include/filtered_tdma_cuda.hpp:152-153).  A is the sub-,
 * B the main- and C the super-diagonal, D the right-hand side.
 *
 * Methods (the reference's backend strings, apps/heat_gpu/tdma_backend_gpu.cu:6-13):
 *   BTDMA_PASCAL       "pascal" | "pascal_tdma"   exact; P segments per system
 *                      with an exact reduced 2P-row interface solve
 *                      (PaScaLTDMACUDA, libs/pascal_tdma/gpu/pascal_tdma_cuda.cu)
 *   BTDMA_FILTERED_V1  "filtered" (any other string)  P segments, adjacent 2x2
 *                      interface solves, J-truncated correction with J taken after
 *                      the interface solve (FilteredTDMACUDA::solve_filtered_v1)
 *   BTDMA_FILTERED_V2  "filtered_v2"  J taken before the sweeps
 *                      (FilteredTDMACUDA::solve_filtered_v2).  Where the P
 *                      segments are whole power-of-two groups of 16-row
 *                      sub-segments (n_row / (16 P) = 1, 2, 4 ... and n_row <=
 *                      512) it runs on the register-tiled kernels: each segment
 *                      solved exactly, the 2x2 interface solves between
 *                      segments, the correction applied in full (no J row
 *                      cut-off: every row is back-substituted anyway); within
 *                      Filtered's eps of PaScaL and of the reference's Filtered,
 *                      at the speed of the tiled PaScaL.  Other shapes, and
 *                      BTDMA_FLAG_REFERENCE_ORDER, run the reference's scheme.
 *   Filtered full-solve fallback: where the reference's truncation gives no
 *   saving or no bound — J >= m - 2 in some segment of m rows (J = m - 1 is
 *   also what the reference sets for rho = 0 or rho >= 0.5,
 *   libs/filtered_tdma/gpu/filtered_tdma_kernels.cuh:245-250) — the reference
 *   still solves the interfaces by the 2x2 approximation; here the batch is
 *   solved with the exact reduced system instead (PaScaL), decided on the
 *   device, and btdma_last_stats reports it (filtered_exact).  With
 *   BTDMA_FLAG_REFERENCE_ORDER the reference's behaviour is kept, bit for bit.
 * With P = 1 every method is the serial Thomas algorithm, bit-identical to the
 * reference's tdma_many / tdma_cyclic_many (libs/pascal_tdma/cpu/tdma_local.cpp),
 * exactly as the reference falls back at nprocs == 1.  In the reference P is the
 * number of MPI ranks a system is split over; here the P segments of a system
 * live in the P CTAs of one thread-block cluster on one GPU.
 *
 * Semantics that differ from the reference's:
 *   - D <- x.  A, B and C are left unchanged (the reference leaves elimination
 *     scratch in A and C).
 *   - Every segment needs >= 3 rows (the reference's PaScaL is wrong at 2,
 *     and indexes out of bounds at 1); btdma_create rejects such a P.
 *   - Calls are stream-ordered and never synchronise the host, except
 *     btdma_last_J and btdma_status, which read back device values, and a
 *     btdma_solve_host call that (re)allocates its staging buffers.
 *
 * Return value of every function: 0 on success, a negative BTDMA_ERR_* code
 * otherwise.  Kernels never trap: runtime faults of the data (NaN/Inf solution,
 * a wait that timed out) are OR-ed into a device status word read by
 * btdma_status().
 */
#ifndef BTDMA_H
#define BTDMA_H

#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct btdma_handle* btdma_t;

enum btdma_method {
    BTDMA_PASCAL = 0,
    BTDMA_FILTERED_V1 = 1,
    BTDMA_FILTERED_V2 = 2
};

enum btdma_precision {
    BTDMA_FP64 = 0,        /* FP64 storage and arithmetic */
    BTDMA_FP32_REFINE = 1, /* FP32 storage, FP32 sweeps + FP64 iterative refinement */
    BTDMA_FP32_STORE = 2   /* FP32 storage widened exactly to FP64, FP64 arithmetic */
};

enum btdma_flags {
    /* Filtered J estimator of the reference's CPU library instead of its CUDA
     * library: v2 takes max|D| over every row of a segment
     * (libs/filtered_tdma/cpu/filtered_tdma.cpp:75-80) instead of its first and
     * last rows (libs/filtered_tdma/gpu/filtered_tdma_kernels.cuh:235-238); v1
     * uses the K bound (filtered_tdma.cpp:110-114) instead of the right-hand-side
     * bound on the post-interface rows (filtered_tdma_cuda.cu:127-131). */
    BTDMA_FLAG_J_HOST = 1 << 0,
    /* PaScaL with the reference's operation order: P cluster CTAs per system,
     * bit-identical to PaScaLTDMA::solve with nprocs = P
     * (libs/pascal_tdma/cpu/pascal_tdma.cpp:113-227).  Without the flag PaScaL
     * uses the register-tiled kernel, exact to rounding (<= 1e-12 relative to
     * the serial Thomas) and faster.  For Filtered handles the flag runs the
     * reference's scheme in its operation order (segment kernels, J-row
     * cut-off) and keeps its 2x2 interface where J >= m - 2 (no exact
     * fallback), so every Filtered result is bit-identical to the
     * reference's. */
    BTDMA_FLAG_REFERENCE_ORDER = 1 << 1
};

enum btdma_error {
    BTDMA_OK = 0,
    BTDMA_ERR_ARG = -1,        /* invalid argument (null handle/pointer, bad size) */
    BTDMA_ERR_SEGMENT = -2,    /* a segment would have fewer than 3 rows */
    BTDMA_ERR_CUDA = -3,       /* a CUDA runtime call failed */
    BTDMA_ERR_SIZE = -4,       /* n_sys / n_row above the handle's capacity */
    BTDMA_ERR_UNSUPPORTED = -5,/* combination not provided (message via btdma_last_error) */
    BTDMA_ERR_DEVICE = -6      /* device status word non-zero (see btdma_status) */
};

/* Create a solver for batches of up to n_sys systems of n_row rows, split into
 * P segments (P = 0 picks P from the shape).  Replaces the constructors
 * PaScaLTDMACUDA(n_sys, myrank, nprocs, comm, block_x, block_y)
 * (libs/pascal_tdma/include/pascal_tdma_cuda.hpp:20-21) and
 * FilteredTDMACUDA(n_sys, n_row, myrank, nprocs, comm, left, right, eps_constant)
 * (libs/filtered_tdma/include/filtered_tdma_cuda.hpp:163-166), with nprocs -> P.
 * Allocates the handle's device scratch; no allocation happens in a solve
 * (btdma_solve_host allocates its staging buffers on first use). */
int btdma_create(int method, int n_sys, int n_row, int P, int precision, int flags,
                 btdma_t* out);

/* Release the handle and its device memory (the reference destructors,
 * pascal_tdma_cuda.cu:153-173, filtered_tdma_cuda.cu:34-54). */
int btdma_destroy(btdma_t h);

/* Solve in place: D <- x.  Replaces PaScaLTDMACUDA::solve(d_A,d_B,d_C,d_D,n_sys,n_row)
 * (pascal_tdma_cuda.hpp:28-29) and FilteredTDMACUDA::solve_filtered_v1/v2(d_A,d_B,d_C,d_D)
 * (filtered_tdma_cuda.hpp:173-174).  n_sys and n_row may be smaller than at
 * create time (n_row must still give every segment >= 3 rows). */
int btdma_solve(btdma_t h, const double* A, const double* B, const double* C, double* D,
                int n_sys, int n_row, cudaStream_t stream);

/* Periodic systems (row 0 couples to row n_row-1 through A[0] and C[n_row-1]).
 * Replaces PaScaLTDMACUDA::solve_cyclic (pascal_tdma_cuda.hpp:32-33) and
 * FilteredTDMACUDA::solve_cycl_filtered_v1/v2 (filtered_tdma_cuda.hpp:179-180). */
int btdma_solve_cyclic(btdma_t h, const double* A, const double* B, const double* C, double* D,
                       int n_sys, int n_row, cudaStream_t stream);

/* Out-of-place solve: X <- x, D unchanged (X may equal D).  No reference
 * counterpart; same kernels as btdma_solve. */
int btdma_solve_out(btdma_t h, const double* A, const double* B, const double* C,
                    const double* D, double* X, int n_sys, int n_row, int cyclic,
                    cudaStream_t stream);

/* Out-of-place solve of a batch in HOST memory: hA, hB, hC, hD, hX are host
 * arrays [n_row x n_sys] (pinned for the copies to overlap; pageable memory
 * works, without overlap).  No reference counterpart: the reference's callers
 * copy to the device themselves (cudaMemcpy) and call solve.  The batch moves
 * in chunks of systems through two device buffer sets that the handle
 * allocates on first use (5 arrays of about n_sys / 8 systems each, kept until
 * btdma_destroy or a larger call): the copy-in of one chunk, the solve of the
 * previous one and the copy-out of the one before overlap on the GPU's two
 * copy engines.  PaScaL chunks solve exactly as a whole-batch btdma_solve_out;
 * Filtered batches go through as one chunk (their truncation depth depends on
 * the whole batch).  Stream-ordered on `stream`: hX is complete once `stream`
 * reaches this point; successive calls on one handle are serialised.  FP64
 * handles only. */
int btdma_solve_host(btdma_t h, const double* hA, const double* hB, const double* hC,
                     const double* hD, double* hX, int n_sys, int n_row, int cyclic,
                     cudaStream_t stream);

/* FP32-stored batch (A, B, C, D float [n_row x n_sys]) solved into an FP64 x:
 * X <- x, 24 bytes of HBM traffic per row instead of 40.  The reference has no
 * FP32 path; the result is compared with the FP64 solve of the same values
 * widened exactly to double.  Handles created with BTDMA_FP32_STORE (FP64
 * arithmetic on the widened values, no refinement needed) or BTDMA_FP32_REFINE
 * (FP32 elimination, FP64 residual and correction sweeps).  PaScaL only; needs
 * n_row a multiple of 16 and n_sys a multiple of 4 (the tiled kernel). */
int btdma_solve_f32(btdma_t h, const float* A, const float* B, const float* C, const float* D,
                    double* X, int n_sys, int n_row, int cyclic, cudaStream_t stream);

/* Filtered: eps = eps_constant / (m * P)^2 per segment of m rows.  Replaces
 * FilteredTDMACUDA::set_eps_constant (filtered_tdma_cuda.hpp:203-206); no-op for
 * PASCAL, as in TdmaBackendGPU::set_eps_constant (tdma_backend_gpu.cu:64-66). */
int btdma_set_eps_constant(btdma_t h, double eps_constant);

/* Filtered: per-row spectral bounds |A_k/B_k|, |C_k/B_k| from system 0's column,
 * stream-ordered on the device.  Replaces FilteredTDMACUDA::set_rho_device
 * (filtered_tdma_cuda.hpp:212; kernel k_set_rho, filtered_tdma_kernels.cuh:46-67).
 * No-op for PASCAL. */
int btdma_set_rho(btdma_t h, const double* A, const double* B, const double* C, int n_sys,
                  int n_row, cudaStream_t stream);

/* Filtered: per-row bounds as the maximum over ALL systems (a conservative
 * estimate for batches whose systems differ; no reference counterpart). */
int btdma_set_rho_all(btdma_t h, const double* A, const double* B, const double* C, int n_sys,
                      int n_row, cudaStream_t stream);

/* Filtered: J of every segment from the most recent solve (blocking device->host
 * read, like FilteredTDMACUDA::last_J, filtered_tdma_cuda.cu:83-87).  Writes
 * min(P, cap) values; returns the number of segments through *n_out. */
int btdma_last_J(btdma_t h, int* J, int cap, int* n_out);

/* Device status word OR-ed by the kernels since the last call (blocking read;
 * resets it to 0).  Bit 0: a wait timed out; bit 1: a non-finite solution. */
int btdma_status(btdma_t h, unsigned* status);

/* Iterative refinement (BTDMA_FP32_REFINE handles): at most max_sweeps
 * correction sweeps (0..BTDMA_REFINE_MAX_SWEEPS, default 3); a system has
 * converged when its normwise backward error
 *     max|D - T x| / (max_j(|A_j| + |B_j| + |C_j|) * max|x| + max|D|)
 * is at most eta_tol (default 8 * 2^-53 ~ 8.9e-16; the forward error is then at
 * most cond(T) * eta_tol).  Systems still above it after the last sweep make
 * the whole batch fall back to the FP64-arithmetic solve of BTDMA_FP32_STORE.
 * No reference counterpart. */
#define BTDMA_REFINE_MAX_SWEEPS 4
int btdma_set_refine(btdma_t h, int max_sweeps, double eta_tol);

/* Statistics of the most recent solve (blocking device->host read).
 * For FP32_REFINE solves: converged_after[k] = systems that met the bound after
 * k corrections (k = 0: the FP32 solve alone), n_fallback = systems that did not
 * meet it after the last sweep (the batch was then solved again with FP64
 * arithmetic), sweeps = correction sweeps that ran.  Other solves report zeros
 * except n_systems.  Replaces nothing in the reference; the counterpart of its
 * J report for the refinement path. */
typedef struct btdma_stats {
    int n_systems;
    int sweeps;
    int converged_after[BTDMA_REFINE_MAX_SWEEPS + 1];
    int n_fallback;
    /* Filtered solves (P > 1): 1 when the batch was solved with the exact
     * reduced system instead of the Filtered interface (see BTDMA_FILTERED_V1),
     * 0 when the Filtered scheme ran; -1 for other solves. */
    int filtered_exact;
} btdma_stats;
int btdma_last_stats(btdma_t h, btdma_stats* stats);

/* Ragged batch: n_sys systems of different lengths stored back to back, system
 * i in rows [row_offsets[i], row_offsets[i+1]) of A, B, C, D (contiguous; the
 * CSR layout), solved by PaScaL with one group of lanes per system into X
 * (X may equal D).  row_offsets (n_sys + 1 entries, starting at 0) and
 * is_periodic (n_sys flags, or NULL for none) are HOST arrays: the first call
 * with a new layout builds a plan (buckets of similar length, device copies of
 * the offsets) and later calls with the same layout reuse it, so build it
 * before capturing a graph.  Every system needs >= 3 rows.  Periodic systems
 * couple row 0 and the last row through A[first] and C[last]; non-periodic ones
 * ignore those two entries.  The _f32 form takes FP32-stored arrays (handle
 * precision FP32_STORE or FP32_REFINE) and computes in FP64 on the widened
 * values.  PaScaL handles only.  The reference solves one uniform batch per
 * call; this replaces looping its solve over equal-length groups. */
int btdma_solve_ragged(btdma_t h, const double* A, const double* B, const double* C,
                       const double* D, double* X, const long long* row_offsets,
                       const unsigned char* is_periodic, int n_sys, cudaStream_t stream);
int btdma_solve_ragged_f32(btdma_t h, const float* A, const float* B, const float* C,
                           const float* D, double* X, const long long* row_offsets,
                           const unsigned char* is_periodic, int n_sys, cudaStream_t stream);

/* Autotuner of ragged solves: times, for every bucket of the plan, each launch
 * shape — P lanes of a warp per system (P = 1..32) with 1..8 warps per CTA, or
 * one CTA of P = 64..512 threads per system (<= 16 rows per thread) — with at
 * least 3 rows per thread, and for non-periodic buckets the interleaved layout
 * (gather into a padded row-interleaved batch, tiled solve, scatter back), on
 * this batch, and keeps the fastest for later solves of the same layout.  Then it times whole
 * solves — every CTA-kind shape as a launch of its own, or the CTA-kind
 * buckets of at most 256 threads in one persistent launch (CTAs split into
 * groups of their buckets' thread counts, taking systems longest first from a
 * counter, then warp-kind tasks of at most 16 rows a lane) — each with the
 * CTA-kind buckets staged as tuned, all staged or all unstaged, and keeps the
 * fastest plan.
 * A..D are double or float as the handle's precision says; X is overwritten.
 * Blocking (it synchronises the stream). */
int btdma_ragged_autotune(btdma_t h, const void* A, const void* B, const void* C, const void* D,
                          double* X, const long long* row_offsets,
                          const unsigned char* is_periodic, int n_sys, cudaStream_t stream);

/* The buckets of the current ragged plan and their launch shapes. */
typedef struct btdma_ragged_bucket {
    int periodic;
    int n_systems;
    int n_row_min, n_row_max;
    int lanes_per_system; /* threads that share one system */
    int warps_per_cta;
    int cta_per_system;   /* 0: lanes of a warp per system; 1: one CTA per system
                             (long systems); 2: one CTA per system staged through
                             shared memory; 3: interleaved layout -- the bucket's
                             systems copied into a row-interleaved batch padded to
                             its longest system (identity rows), solved by the
                             tiled kernel and copied back (non-periodic buckets,
                             lanes_per_system 1) */
    float tuned_ms;       /* fastest time measured by the autotuner (0 before tuning) */
    int persistent;       /* 1: the bucket's systems run in the plan's one persistent
                             launch (CTA-kind buckets of at most 256 threads, when the
                             autotuner measured that faster than a launch per
                             shape); 0: a launch of its own shape */
} btdma_ragged_bucket;
int btdma_ragged_plan_info(btdma_t h, btdma_ragged_bucket* out, int cap, int* n_out);

/* Replace the launch shapes of the current ragged plan (lanes_per_system and
 * cta_per_system of every bucket, and the persistent launch when any bucket's
 * persistent is set; the other fields must match the plan, in plan_info's
 * order): restores a plan tuned earlier, e.g. by another process,
 * without timing again.  Every shape is checked against the limits the
 * autotuner uses (P a power of two, >= 3 rows per thread, per-thread row and
 * shared-memory caps); a rejected plan leaves the current one in place.  No
 * counterpart in the reference. */
int btdma_ragged_set_plan(btdma_t h, const btdma_ragged_bucket* buckets, int n);

/* Fused 3-D heat ADI step: the theta-scheme step of the reference's heat
 * application (apps/heat_gpu/solve_theta.cu, SolveTheta::profile's step loop:
 * ghost fill, right-hand side, Z, Y and X sweeps with fully implicit Dirichlet
 * walls, update) on ix x iy x iz interior cells of [-1, 1]^3, one GPU, PaScaL
 * solves.  theta is the caller's device field with one ghost layer,
 * theta[(k * (iy + 2) + j) * (ix + 2) + i].  Each sweep's tridiagonal
 * coefficients are generated inside the solve (never stored); ix, iy, iz must
 * be multiples of 16.  btdma_heat_step runs n_steps steps, as one captured
 * CUDA graph replayed per step when use_graph != 0 (captured on the first call
 * for this theta pointer).  btdma_heat_init writes the reference's initial
 * field; btdma_heat_l2_error returns the reference's global L2 error against
 * the manufactured solution at physical time t_phys (sum over interior cells
 * divided by (ix + 1)(iy + 1)(iz + 1), heat_cpu/main.cpp:59-79; blocking). */
typedef struct btdma_heat* btdma_heat_t;
int btdma_heat_create(int ix, int iy, int iz, double dt, btdma_heat_t* out);
int btdma_heat_destroy(btdma_heat_t h);
int btdma_heat_init(btdma_heat_t h, double* theta, cudaStream_t stream);
int btdma_heat_step(btdma_heat_t h, double* theta, int n_steps, int use_graph,
                    cudaStream_t stream);
int btdma_heat_l2_error(btdma_heat_t h, const double* theta, double t_phys, double* l2);
/* One step launched phase by phase with CUDA events between the phases
 * (blocking); writes the 12 per-step times in seconds of the reference's timing
 * events, in its order (solve_theta.cu:436-439): rhs, solve_z, solve_y,
 * solve_x, etc, comm, tdma_z_comm, tdma_y_comm, tdma_x_comm, tdma_z_gpu,
 * tdma_y_gpu, tdma_x_gpu.  solve_d spans a sweep's solve and the re-layout that
 * follows it; etc, comm and the *_comm events are 0 (one GPU, ghosts computed
 * in the right-hand-side kernel). */
int btdma_heat_step_profile(btdma_heat_t h, double* theta, double* times, cudaStream_t stream);

/* Wall-normal solve of the channel flow's FFT Poisson equation: for every
 * Fourier mode m (n_modes of them) and row k = 0..nz-1,
 *     a_k p_{k-1} - (a_k + c_k + lambda_m) p_k + c_k p_{k+1} = rhs_k,
 *     a_k = 1 / (dz[k+1] dmz[k+1]) (0 for k = 0),
 *     c_k = 1 / (dz[k+1] dmz[k+2]) (0 for k = nz - 1),
 * solved for the real and imaginary parts of the complex right-hand side with
 * one set of coefficients (replaces k_build_poisson_tdma + two TDMA solves of
 * PressureSolverGPU::solve_tdma_z_, PressureSolverGPU.cu:183-220 and
 * :514-537, which store every coefficient twice).  With pin_mode0, row 0 of
 * mode 0 becomes p_0 = 0 (k_zero_mode).  dz and dmz (nz + 2 entries, ghosts
 * included) and lambda (n_modes, kx^2 + ky^2 of each mode) are HOST arrays read
 * at create time.  rhs is the device complex array [nz][n_modes] as
 * interleaved (real, imaginary) doubles (the reference's hat_Y layout with
 * mode = j * nxh + i), overwritten with the solution.  nz must be a multiple
 * of 16; coefficients are generated inside the solve, never stored. */
typedef struct btdma_poisson* btdma_poisson_t;
int btdma_poisson_create(int nz, const double* dz, const double* dmz, int n_modes,
                         const double* lambda, int pin_mode0, btdma_poisson_t* out);
int btdma_poisson_destroy(btdma_poisson_t h);
int btdma_poisson_solve(btdma_poisson_t h, double* rhs, cudaStream_t stream);
int btdma_poisson_status(btdma_poisson_t h, unsigned* status, cudaStream_t stream);

/* Channel momentum ADI sweeps (apps/channel_gpu/MomentumSolverGPU.cu: adi_z_,
 * adi_y_, adi_x_ at :261-313 with k_build_* / k_scatter_* at :135-220): the
 * implicit viscous half-step of velocity component comp (0 u, 1 v, 2 w) along
 * direction dir (0 x, 1 y, 2 z) on an nx x ny x nz grid, field
 * q[i + (nx+2) * (j + (ny+2) * k)] with one ghost layer.  Row r of a sweep is
 *     -c ar_r x_{r-1} + (1 + c (ar_r + cr_r)) x_r - c cr_r x_{r+1} = q_r
 * with ar, cr from the cell sizes dx and centre spacings dmx of that axis
 * (staggered when comp == dir), no-slip walls at both z ends (u, v: the
 * ghost folded onto the diagonal; w: w = 0 on the first face) and periodic x
 * / y sweeps when pbc_x / pbc_y.  dx*, dmx* are HOST arrays of n + 2 entries
 * (ghosts included), read at create time.  Coefficients are generated inside
 * the solve, never stored.  btdma_momentum_sweep reads q and writes dst (may
 * be q); btdma_momentum_adi runs the z, y and x sweeps of
 * MomentumSolverGPU::advance's diffuse step after k_lap and writes the result
 * into q_out's interior.  With the default (PaScaL) backend it only reads
 * rhs: each sweep stores its solution straight into the next sweep's layout
 * (four kernels); with a Filtered backend it runs the reference's sequence, z
 * and y in place on rhs.  PaScaL (exact)
 * solves; n a multiple of 16, n / 16 a power of two for periodic sweeps.  The
 * handle keeps each (dir, comp) factor table until c or the stream changes;
 * a sweep captured into a CUDA graph builds its table on every replay, into a
 * second set of tables kept for captured sweeps, so replays never change what
 * uncaptured calls reuse.  Calls and graph replays on one handle must be
 * ordered (one stream, or synchronised). */
typedef struct btdma_momentum* btdma_momentum_t;
int btdma_momentum_create(int nx, int ny, int nz, const double* dx0, const double* dmx0,
                          const double* dx1, const double* dmx1, const double* dx2,
                          const double* dmx2, int pbc_x, int pbc_y, btdma_momentum_t* out);
int btdma_momentum_destroy(btdma_momentum_t h);
int btdma_momentum_sweep(btdma_momentum_t h, int dir, int comp, const double* q, double* dst,
                         double c, cudaStream_t stream);
int btdma_momentum_adi(btdma_momentum_t h, int comp, double* rhs, double* q_out, double c,
                       cudaStream_t stream);
int btdma_momentum_status(btdma_momentum_t h, unsigned* status, cudaStream_t stream);

/* Solver of the momentum sweeps: BTDMA_PASCAL (the default: the tiled exact
 * solve with generated coefficients above), or BTDMA_FILTERED_V1 / _V2 with P
 * segments per system, the backend string of the reference's channel solver
 * (TdmaSolverGPU::parse_backend: anything but "pascal" selects
 * FilteredTDMACUDA::solve_[cycl_]filtered_v2; apps/channel_gpu/
 * TdmaSolverGPU.cpp:10-17, 37-51).  With a Filtered method every sweep runs the
 * reference's sequence (MomentumSolverGPU::adi_{z,y,x}_, :261-313): A, B, C, D
 * built into arrays in k_build_{x,y,z}'s arithmetic, rho from system 0's
 * column (set_rho_device), the solve of a library handle of that method, P and
 * flags (btdma_create; eps_constant as set_eps_constant, the reference passes
 * dt), periodic x / y sweeps by the cyclic solve, then the scatter.  P = 1 is
 * the serial Thomas algorithm, bit-identical to the reference's one-rank
 * channel run with either backend.  Allocates four field-sized arrays on
 * first use.  No counterpart of its own in the reference. */
int btdma_momentum_set_backend(btdma_momentum_t h, int method, int P, int flags,
                               double eps_constant);

/* Self test of the failure path of every pipeline wait: a one-thread kernel
 * waits with each of the library's bounded waits (at most `limit` polls; a
 * hinted poll lasts up to 20 us, an unhinted one far less) on an mbarrier
 * nothing arrives at; *status_out receives the AND of their device status
 * words, which must have BTDMA_STATUS_TIMEOUT set.  No fault, no hang. */
#define BTDMA_STATUS_TIMEOUT 1u
#define BTDMA_STATUS_NONFINITE 2u
int btdma_selftest_wait_timeout(int limit, unsigned* status_out, cudaStream_t stream);

/* Switch the method of an existing handle (rho, eps and J state are kept).  The
 * reference's FilteredTDMACUDA object offers v1 and v2 side by side
 * (filtered_tdma_cuda.hpp:173-180); this lets one handle do the same. */
int btdma_set_method(btdma_t h, int method);

/* Segments per system used by the handle (after the P = 0 choice). */
int btdma_segments(btdma_t h, int* P);

/* Kernel shape of the PaScaL solves that run the register-tiled kernel
 * (FP64 and FP32 storage with FP64 arithmetic).  NARROW: SYS systems per CTA
 * with every row's elimination state in registers.  WIDE: twice the systems
 * per CTA (wider HBM row pieces), half of each group's rows read a second time
 * from L2 instead of held.  AUTO: the library's measured choice per shape.
 * Both return the same bits.  No counterpart in the reference. */
enum btdma_tile_shape {
    BTDMA_TILE_AUTO = 0,
    BTDMA_TILE_NARROW = 1,
    BTDMA_TILE_WIDE = 2
};
int btdma_set_tile_shape(btdma_t h, int shape);

/* Serial Thomas solve (D <- x, bit-identical to btdma_solve with P = 1) that
 * allocates nothing.  No counterpart in the reference.
 *
 * For callers that must not allocate device memory: code running under a
 * framework that owns the GPU memory pool, loops that cannot afford an
 * allocation's latency or its implicit synchronisation, and places where
 * CUDA's allocation calls are not allowed at all.  There is no handle; the
 * elimination scratch is a fixed array inside the library, BTDMA_NOALLOC_MAX_ELEMS
 * doubles (8 MiB) that every GPU loading the library keeps until the process
 * exits.  Batches with n_sys * n_row above that return BTDMA_ERR_SIZE.
 *
 * The first call on a device (and the first after that device's context was
 * destroyed and created again) looks up the array's device address in the
 * current context; make that first call before any stream capture.  All
 * calls share the one array and leave their
 * scratch in it, so calls that overlap on the GPU (other streams, other host
 * threads) race with each other: order them on one stream.  A, B, C are
 * unchanged; no device status word is kept. */
#define BTDMA_NOALLOC_MAX_ELEMS (1 << 20)
int btdma_solve_noalloc(const double* A, const double* B, const double* C, double* D,
                        int n_sys, int n_row, cudaStream_t stream);

/* Message of the most recent failing call on this thread. */
const char* btdma_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* BTDMA_H */
