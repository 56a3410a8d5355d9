// Driver for the reference's own CPU solver library, built from its sources —
// TEST INFRASTRUCTURE ONLY (checker and CPU baseline; never the product path).
//
// Links the unmodified reference files
//   libs/pascal_tdma/cpu/{tdma_local.cpp, pascal_tdma.cpp, para_range.cpp}
//   libs/filtered_tdma/cpu/{tdma_local.cpp, filtered_tdma.cpp, filtered_tdma_profile.cpp}
// against the thread-rank MPI stand-in in mpi_shim/.  Each entry point takes a
// whole batch in the reference layout [n_row x n_sys] (row j at j*n_sys), splits
// the rows over `nprocs` thread ranks with the reference's para_range block split
// (libs/pascal_tdma/cpu/para_range.cpp:4-10), runs one reference solver object per
// rank exactly as its apps do (apps/heat_cpu/tdma_backend.cpp:16-31, 54-75), and
// gathers the rows back.

#include <mpi.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "pascal_tdma.hpp"
#include "filtered_tdma.hpp"

void tdma_many(double*, double*, double*, double*, int, int);
void tdma_cyclic_many(double*, double*, double*, double*, int, int);
void ftdma_many(double*, double*, double*, double*, int, int);
void ftdma_cyclic_many(double*, double*, double*, double*, int, int);
void para_range(int start, int end, int nproc, int rank, int& ista, int& iend);

namespace {

struct Slab {
    int row0, nrow;
    std::vector<double> A, B, C, D;
};

std::vector<Slab> split_rows(const double* A, const double* B, const double* C,
                             const double* D, int n_sys, int n_row, int nprocs) {
    std::vector<Slab> s(nprocs);
    for (int p = 0; p < nprocs; ++p) {
        int ista, iend;
        para_range(0, n_row - 1, nprocs, p, ista, iend);
        s[p].row0 = ista;
        s[p].nrow = iend - ista + 1;
        size_t off = (size_t)ista * n_sys, cnt = (size_t)s[p].nrow * n_sys;
        s[p].A.assign(A + off, A + off + cnt);
        s[p].B.assign(B + off, B + off + cnt);
        s[p].C.assign(C + off, C + off + cnt);
        s[p].D.assign(D + off, D + off + cnt);
    }
    return s;
}

void gather_rows(const std::vector<Slab>& s, double* A, double* C, double* D, int n_sys) {
    for (const Slab& sl : s) {
        size_t off = (size_t)sl.row0 * n_sys;
        std::copy(sl.A.begin(), sl.A.end(), A + off);
        std::copy(sl.C.begin(), sl.C.end(), C + off);
        std::copy(sl.D.begin(), sl.D.end(), D + off);
    }
}

template <class F>
void run_ranks(int nprocs, F&& body) {
    MPI_Comm comm = shim_comm_create(nprocs);
    std::vector<std::thread> th;
    for (int p = 0; p < nprocs; ++p)
        th.emplace_back([&, p] {
            shim_bind_rank(comm, p);
            body(p, comm);
        });
    for (auto& t : th) t.join();
    shim_comm_destroy(comm);
}

// Per-row spectral bounds from system 0's column, as the reference's CPU backend
// does before each Filtered solve (apps/heat_cpu/tdma_backend.cpp:33-44).  When
// `rho_row` is given, row k of the global system uses rho_row[k] for both.
void fill_rho(FilteredTDMA& f, const Slab& sl, int n_sys, const double* rho_row) {
    std::vector<double>& ar = f.A_rho();
    std::vector<double>& cr = f.C_rho();
    for (int k = 0; k < sl.nrow; ++k) {
        if (rho_row) {
            ar[k] = cr[k] = rho_row[sl.row0 + k];
        } else {
            double b = sl.B[(size_t)k * n_sys];
            ar[k] = b != 0.0 ? std::fabs(sl.A[(size_t)k * n_sys] / b) : 0.0;
            cr[k] = b != 0.0 ? std::fabs(sl.C[(size_t)k * n_sys] / b) : 0.0;
        }
    }
    ar[sl.nrow] = 0.0;
    cr[sl.nrow] = 0.0;
}

}  // namespace

extern "C" {

void ref_tdma_many(double* A, double* B, double* C, double* D, int n_sys, int n_row) {
    tdma_many(A, B, C, D, n_sys, n_row);
}
void ref_ftdma_many(double* A, double* B, double* C, double* D, int n_sys, int n_row) {
    ftdma_many(A, B, C, D, n_sys, n_row);
}
void ref_tdma_cyclic_many(double* A, double* B, double* C, double* D, int n_sys, int n_row) {
    tdma_cyclic_many(A, B, C, D, n_sys, n_row);
}
void ref_ftdma_cyclic_many(double* A, double* B, double* C, double* D, int n_sys, int n_row) {
    ftdma_cyclic_many(A, B, C, D, n_sys, n_row);
}
void ref_para_range(int start, int end, int nproc, int rank, int* ista, int* iend) {
    para_range(start, end, nproc, rank, *ista, *iend);
}

// PaScaLTDMA::solve / solve_cyclic with `nprocs` thread ranks.
void ref_pascal(double* A, double* B, double* C, double* D, int n_sys, int n_row,
                int nprocs, int cyclic) {
    std::vector<Slab> s = split_rows(A, B, C, D, n_sys, n_row, nprocs);
    run_ranks(nprocs, [&](int p, MPI_Comm comm) {
        PaScaLTDMA solver(n_sys, p, nprocs, comm);
        Slab& sl = s[p];
        if (cyclic)
            solver.solve_cyclic(sl.A.data(), sl.B.data(), sl.C.data(), sl.D.data(), n_sys, sl.nrow);
        else
            solver.solve(sl.A.data(), sl.B.data(), sl.C.data(), sl.D.data(), n_sys, sl.nrow);
    });
    gather_rows(s, A, C, D, n_sys);
}

// FilteredTDMA::solve_[cycl_]filtered_v{1,2} with `nprocs` thread ranks.
void ref_filtered(double* A, double* B, double* C, double* D, int n_sys, int n_row,
                  int nprocs, int version, int cyclic, double eps_constant,
                  const double* rho_row) {
    std::vector<Slab> s = split_rows(A, B, C, D, n_sys, n_row, nprocs);
    run_ranks(nprocs, [&](int p, MPI_Comm comm) {
        Slab& sl = s[p];
        int left = p - 1, right = p + 1;
        if (cyclic) {
            left = (p - 1 + nprocs) % nprocs;
            right = (p + 1) % nprocs;
        } else {
            if (left < 0) left = MPI_PROC_NULL;
            if (right >= nprocs) right = MPI_PROC_NULL;
        }
        FilteredTDMA f(n_sys, sl.nrow, p, nprocs, comm, left, right, eps_constant);
        fill_rho(f, sl, n_sys, rho_row);
        double *a = sl.A.data(), *b = sl.B.data(), *c = sl.C.data(), *d = sl.D.data();
        if (version == 1)
            cyclic ? f.solve_cycl_filtered_v1(a, b, c, d) : f.solve_filtered_v1(a, b, c, d);
        else
            cyclic ? f.solve_cycl_filtered_v2(a, b, c, d) : f.solve_filtered_v2(a, b, c, d);
    });
    gather_rows(s, A, C, D, n_sys);
}

// CPU baseline: time `reps` PaScaLTDMA solves (method 0) or Filtered v2 solves
// (method 2) of one batch with `nprocs` thread ranks, each rank holding its slab
// of rows.  The inputs are restored from a pristine copy outside the timed
// region.  Each entry of `seconds` is the max over ranks of one solve.
void ref_time_solve(const double* A, const double* B, const double* C, const double* D,
                    int n_sys, int n_row, int nprocs, int method, double eps_constant,
                    int reps, double* seconds) {
    std::vector<Slab> pristine = split_rows(A, B, C, D, n_sys, n_row, nprocs);
    std::vector<Slab> work = pristine;
    std::vector<double> t(nprocs * reps, 0.0);
    run_ranks(nprocs, [&](int p, MPI_Comm comm) {
        Slab& sl = work[p];
        const Slab& pr = pristine[p];
        PaScaLTDMA* pas = nullptr;
        FilteredTDMA* fil = nullptr;
        if (method == 0) {
            pas = new PaScaLTDMA(n_sys, p, nprocs, comm);
        } else {
            int left = p > 0 ? p - 1 : MPI_PROC_NULL;
            int right = p + 1 < nprocs ? p + 1 : MPI_PROC_NULL;
            fil = new FilteredTDMA(n_sys, sl.nrow, p, nprocs, comm, left, right, eps_constant);
            fill_rho(*fil, pr, n_sys, nullptr);
        }
        for (int r = 0; r < reps; ++r) {
            std::copy(pr.A.begin(), pr.A.end(), sl.A.begin());
            std::copy(pr.C.begin(), pr.C.end(), sl.C.begin());
            std::copy(pr.D.begin(), pr.D.end(), sl.D.begin());
            MPI_Barrier(comm);
            double t0 = MPI_Wtime();
            if (pas)
                pas->solve(sl.A.data(), sl.B.data(), sl.C.data(), sl.D.data(), n_sys, sl.nrow);
            else
                fil->solve_filtered_v2(sl.A.data(), sl.B.data(), sl.C.data(), sl.D.data());
            t[p * reps + r] = MPI_Wtime() - t0;
            MPI_Barrier(comm);
        }
        delete pas;
        delete fil;
    });
    for (int r = 0; r < reps; ++r) {
        double m = 0.0;
        for (int p = 0; p < nprocs; ++p) m = std::max(m, t[p * reps + r]);
        seconds[r] = m;
    }
}

}  // extern "C"
