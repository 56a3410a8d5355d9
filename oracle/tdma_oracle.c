/*
 * CPU oracle for the batched tridiagonal solve — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's algorithms, used only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.  The
 * product library never links or calls it.  It is pinned against the reference's
 * own CPU library built from its sources (oracle/_ref, see Makefile) and against
 * committed golden vectors (tests/golden/).
 *
 * Layout: every array is [n_row x n_sys] row-major, row j of system i at
 * j*n_sys + i (libs/pascal_tdma/include/pascal_tdma.hpp:13).  All arithmetic is
 * FP64 with the operation order of the reference; compile with
 * -ffp-contract=off so that no multiply-add is fused (the reference's CPU build
 * is ISO C++17 with g++, which does not contract: Makefile.inc:24).
 *
 * Segments: a system of n_row rows split into P segments follows the block split
 * of libs/pascal_tdma/cpu/para_range.cpp:4-10 (segment p has base+(p<rem) rows).
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#define AT(arr, j, i) (arr)[(size_t)(j) * n_sys + (i)]

/* libs/pascal_tdma/cpu/para_range.cpp:4-10 over the 0-based range [0, n). */
void orc_split(int n, int nparts, int part, int* first, int* count) {
    int base = n / nparts, rem = n % nparts;
    *first = part * base + (part < rem ? part : rem);
    *count = base + (part < rem ? 1 : 0);
}

/* ---------------------------------------------------------------------------
 * Serial Thomas, libs/pascal_tdma/cpu/tdma_local.cpp:6-52 (tdma_many).
 * C <- forward-eliminated c', D <- x.  A and B are read only.
 * ------------------------------------------------------------------------- */
void orc_thomas(const double* A, const double* B, double* C, double* D,
                int n_sys, int n_row) {
    /* Row sweeps over all systems, as tdma_many's loops (rows outer, systems
     * inner); every system sees exactly the operations of the serial
     * recurrence. */
    for (int i = 0; i < n_sys; ++i) {
        double inv_b = 1.0 / AT(B, 0, i);
        AT(D, 0, i) = AT(D, 0, i) * inv_b;
        AT(C, 0, i) = AT(C, 0, i) * inv_b;
    }
    for (int j = 1; j < n_row; ++j)
        for (int i = 0; i < n_sys; ++i) {
            double a = AT(A, j, i);
            double r = 1.0 / (AT(B, j, i) - a * AT(C, j - 1, i));
            AT(D, j, i) = r * (AT(D, j, i) - a * AT(D, j - 1, i));
            AT(C, j, i) = r * AT(C, j, i);
        }
    for (int j = n_row - 2; j >= 0; --j)
        for (int i = 0; i < n_sys; ++i)
            AT(D, j, i) = AT(D, j, i) - AT(C, j, i) * AT(D, j + 1, i);
}

/* ---------------------------------------------------------------------------
 * Periodic Thomas with the correction vector E,
 * libs/pascal_tdma/cpu/tdma_local.cpp:108-208 (tdma_cyclic_many).
 * Row 0 couples to row n_row-1 through A[0] and C[n_row-1].  Needs n_row >= 3.
 * Systems go in blocks of ORC_BLK, rows outer within a block (E is the
 * block's [n_row x ORC_BLK] workspace).
 * ------------------------------------------------------------------------- */
#define ORC_BLK 256
void orc_thomas_cyclic(const double* A, const double* B, double* C, double* D,
                       int n_sys, int n_row) {
    double* E = (double*)malloc(sizeof(double) * (size_t)n_row * ORC_BLK);
#define EB(j, b) E[(size_t)(j) * ORC_BLK + (b)]
    for (int i0 = 0; i0 < n_sys; i0 += ORC_BLK) {
        const int nb = n_sys - i0 < ORC_BLK ? n_sys - i0 : ORC_BLK;
        for (int b = 0; b < nb; ++b) {
            const int i = i0 + b;
            for (int j = 0; j < n_row; ++j) EB(j, b) = 0.0;
            EB(1, b) = -AT(A, 1, i);
            EB(n_row - 1, b) = -AT(C, n_row - 1, i);
            double inv_b = 1.0 / AT(B, 1, i);
            AT(D, 1, i) = AT(D, 1, i) * inv_b;
            EB(1, b) = EB(1, b) * inv_b;
            AT(C, 1, i) = AT(C, 1, i) * inv_b;
        }
        for (int j = 2; j < n_row; ++j)
            for (int b = 0; b < nb; ++b) {
                const int i = i0 + b;
                double a = AT(A, j, i);
                double r = 1.0 / (AT(B, j, i) - a * AT(C, j - 1, i));
                AT(D, j, i) = r * (AT(D, j, i) - a * AT(D, j - 1, i));
                EB(j, b) = r * (EB(j, b) - a * EB(j - 1, b));
                AT(C, j, i) = r * AT(C, j, i);
            }
        for (int j = n_row - 2; j >= 1; --j)
            for (int b = 0; b < nb; ++b) {
                const int i = i0 + b;
                double c = AT(C, j, i);
                AT(D, j, i) = AT(D, j, i) - c * AT(D, j + 1, i);
                EB(j, b) = EB(j, b) - c * EB(j + 1, b);
            }
        for (int b = 0; b < nb; ++b) {
            const int i = i0 + b;
            double a0 = AT(A, 0, i), c0 = AT(C, 0, i);
            double x0 = (AT(D, 0, i) - a0 * AT(D, n_row - 1, i) - c0 * AT(D, 1, i)) /
                        (AT(B, 0, i) + a0 * EB(n_row - 1, b) + c0 * EB(1, b));
            AT(D, 0, i) = x0;
        }
        for (int j = 1; j < n_row; ++j)
            for (int b = 0; b < nb; ++b) {
                const int i = i0 + b;
                AT(D, j, i) = AT(D, j, i) + AT(D, 0, i) * EB(j, b);
            }
    }
#undef EB
    free(E);
}

/* ---------------------------------------------------------------------------
 * Modified Thomas on one segment (rows r0..r0+m-1 of the batch), the per-rank
 * local steps of libs/pascal_tdma/cpu/pascal_tdma.cpp:131-183:
 *   forward  (rows 0,1 normalised; j>=2 eliminate a, keep coupling to x_0),
 *   backward (j=m-3..1, fold in coupling to x_{m-1}),
 *   row-0 reduction (r = 1/(1 - A1*C0)).
 * Afterwards every interior row j reads  A_j x_0 + x_j + C_j x_{m-1} = D_j,
 * row 0 reads  A_0 x_prev + x_0 + C_0 x_{m-1} = D_0  and row m-1 reads
 * A_{m-1} x_0 + x_{m-1} + C_{m-1} x_next = D_{m-1}.  Needs m >= 3 (the
 * reference's row-0 reduction treats row 1 as interior).
 * ------------------------------------------------------------------------- */
static void modified_thomas_segment(double* A, const double* B, double* C, double* D,
                                    int n_sys, int i, int r0, int m) {
#define S(arr, j) AT(arr, r0 + (j), i)
    double q0 = 1.0 / S(B, 0);
    S(A, 0) = S(A, 0) * q0;
    S(C, 0) = S(C, 0) * q0;
    S(D, 0) = S(D, 0) * q0;
    double q1 = 1.0 / S(B, 1);
    S(A, 1) = S(A, 1) * q1;
    S(C, 1) = S(C, 1) * q1;
    S(D, 1) = S(D, 1) * q1;
    for (int j = 2; j < m; ++j) {
        double a = S(A, j);
        double inv = 1.0 / (S(B, j) - a * S(C, j - 1));
        S(D, j) = inv * (S(D, j) - a * S(D, j - 1));
        S(C, j) = inv * S(C, j);
        S(A, j) = -inv * a * S(A, j - 1);
    }
    for (int j = m - 3; j >= 1; --j) {
        double c = S(C, j);
        S(D, j) = S(D, j) - c * S(D, j + 1);
        S(A, j) = S(A, j) - c * S(A, j + 1);
        S(C, j) = c * -S(C, j + 1);
    }
    double r = 1.0 / (1.0 - S(A, 1) * S(C, 0));
    S(D, 0) = r * (S(D, 0) - S(C, 0) * S(D, 1));
    S(A, 0) = r * S(A, 0);
    S(C, 0) = -r * S(C, 0) * S(C, 1);
#undef S
}

/* ---------------------------------------------------------------------------
 * PaScaL with P segments per system, libs/pascal_tdma/cpu/pascal_tdma.cpp:113-348
 * (solve / solve_cyclic with nprocs = P).  The reduced system has rows
 * (2p, 2p+1) = (first, last) row of segment p, unit diagonal, and is solved by
 * the serial Thomas (tdma_many with B = 1, pascal_tdma.cpp:200-201) or its
 * periodic form (pascal_tdma.cpp:321-322).  The all-to-all transpose of the
 * reference only distributes systems over ranks; per system the arithmetic is
 * this.  D <- x; A and C are overwritten with the segment coefficients.
 * Returns 0, or -1 when some segment has fewer than 3 rows.
 * ------------------------------------------------------------------------- */
int orc_pascal(double* A, const double* B, double* C, double* D,
               int n_sys, int n_row, int P, int cyclic) {
    if (P == 1) {
        if (cyclic)
            orc_thomas_cyclic(A, B, C, D, n_sys, n_row);
        else
            orc_thomas(A, B, C, D, n_sys, n_row);
        return 0;
    }
    for (int p = 0; p < P; ++p) {
        int r0, m;
        orc_split(n_row, P, p, &r0, &m);
        if (m < 3) return -1;
    }
    const int nr = 2 * P;
    double* rA = (double*)malloc(sizeof(double) * nr);
    double* rB = (double*)malloc(sizeof(double) * nr);
    double* rC = (double*)malloc(sizeof(double) * nr);
    double* rD = (double*)malloc(sizeof(double) * nr);
    for (int i = 0; i < n_sys; ++i) {
        for (int p = 0; p < P; ++p) {
            int r0, m;
            orc_split(n_row, P, p, &r0, &m);
            modified_thomas_segment(A, B, C, D, n_sys, i, r0, m);
            rA[2 * p] = AT(A, r0, i);
            rC[2 * p] = AT(C, r0, i);
            rD[2 * p] = AT(D, r0, i);
            rA[2 * p + 1] = AT(A, r0 + m - 1, i);
            rC[2 * p + 1] = AT(C, r0 + m - 1, i);
            rD[2 * p + 1] = AT(D, r0 + m - 1, i);
        }
        for (int k = 0; k < nr; ++k) rB[k] = 1.0;
        /* one-system solve of the reduced rows (n_sys = 1 layout) */
        if (cyclic)
            orc_thomas_cyclic(rA, rB, rC, rD, 1, nr);
        else
            orc_thomas(rA, rB, rC, rD, 1, nr);
        for (int p = 0; p < P; ++p) {
            int r0, m;
            orc_split(n_row, P, p, &r0, &m);
            double x0 = rD[2 * p], xn = rD[2 * p + 1];
            AT(D, r0, i) = x0;
            AT(D, r0 + m - 1, i) = xn;
            for (int j = 1; j < m - 1; ++j)
                AT(D, r0 + j, i) = AT(D, r0 + j, i) -
                                   (AT(A, r0 + j, i) * x0 + AT(C, r0 + j, i) * xn);
        }
    }
    free(rA);
    free(rB);
    free(rC);
    free(rD);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Truncation depth J of the Filtered scheme.
 *   rho   = max over the segment's rows 1..m-1 of the per-row bound
 *           (filtered_tdma.cpp:66-71; the +1 slot of A_rho/C_rho is never read);
 *   rho in {0} u [0.5, inf)  ->  J = m-1  (full propagation);
 *   lambda = (1+sqrt(1-4 rho^2))/2, q = rho/lambda;
 *   rhs bound  B = q(2+q)/((1-q)(1-2 rho)) * max_b     (filtered_tdma.cpp:82-86)
 *   K bound    B = (maxD0 + maxDN) q/(1-q)              (filtered_tdma.cpp:110-114)
 *   J = int(log(eps/B)/log q) + 1, at most m-1; the device estimator also
 *   clamps J >= 0 (filtered_tdma_kernels.cuh:249-257).
 * ------------------------------------------------------------------------- */
static int j_from_bound(double rho, double bound, double eps, int m, int clamp0) {
    if (rho == 0.0 || rho >= 0.5) return m - 1;
    int J = (int)(log(eps / bound) / log(rho / ((1.0 + sqrt(1.0 - 4.0 * rho * rho)) / 2.0))) + 1;
    if (J > m - 1) J = m - 1;
    if (clamp0 && J < 0) J = 0;
    return J;
}

static double q_of(double rho) { return rho / ((1.0 + sqrt(1.0 - 4.0 * rho * rho)) / 2.0); }

double orc_rhs_bound_factor(double rho) {
    double q = q_of(rho);
    return q * (2.0 + q) / ((1.0 - q) * (1.0 - 2.0 * rho));
}

/* J estimator semantics. */
enum {
    ORC_J_DEVICE = 0, /* device estimator: max|D| over the segment's first and last
                         rows (filtered_tdma_kernels.cuh:220-261); v1 evaluates it on
                         the post-interface rows (filtered_tdma_cuda.cu:127-131) */
    ORC_J_HOST = 1    /* host estimator: v2 max|D| over every row of the segment
                         (filtered_tdma.cpp:63-87); v1 uses the K bound on the
                         post-interface rows (filtered_tdma.cpp:89-115) */
};

/* ---------------------------------------------------------------------------
 * Filtered TDMA with P segments per system, filtered_tdma.cpp:170-258 with the
 * steps of filtered_tdma_kernels.hpp:35-250, nprocs = P.  Segment p talks to
 * p-1 and p+1 (and wraps when `cyclic`).  `rho_row[k]` is the per-row bound
 * max(|A_k/B_k|, |C_k/B_k|) of global row k.  eps of segment p is
 * eps_constant / (m_p * P)^2 (filtered_tdma.cpp:49-51).  J of every segment is
 * written to J_out[p] (m-1 when P == 1, where the solve is the serial Thomas).
 * Returns 0, or -1 when some segment has fewer than 3 rows.
 * ------------------------------------------------------------------------- */
int orc_filtered(double* A, const double* B, double* C, double* D,
                 int n_sys, int n_row, int P, int version, int cyclic,
                 double eps_constant, const double* rho_row, int jmode, int* J_out) {
    if (P == 1) {
        if (cyclic)
            orc_thomas_cyclic(A, B, C, D, n_sys, n_row);
        else
            orc_thomas(A, B, C, D, n_sys, n_row);
        if (J_out) J_out[0] = n_row - 1;
        return 0;
    }
    int* r0s = (int*)malloc(sizeof(int) * P);
    int* ms = (int*)malloc(sizeof(int) * P);
    int* Js = (int*)malloc(sizeof(int) * P);
    int* Jrep = (int*)malloc(sizeof(int) * P);
    double* rhos = (double*)malloc(sizeof(double) * P);
    double* eps = (double*)malloc(sizeof(double) * P);
    for (int p = 0; p < P; ++p) {
        orc_split(n_row, P, p, &r0s[p], &ms[p]);
        if (ms[p] < 3) {
            free(r0s); free(ms); free(Js); free(Jrep); free(rhos); free(eps);
            return -1;
        }
        double rho = 0.0;
        for (int k = 1; k < ms[p]; ++k)
            if (rho_row[r0s[p] + k] > rho) rho = rho_row[r0s[p] + k];
        rhos[p] = rho;
        int N = ms[p] * P;
        eps[p] = eps_constant / ((double)N * N);
    }

    /* v2: J before the sweeps, from the pre-solve right-hand side. */
    if (version == 2) {
        for (int p = 0; p < P; ++p) {
            int r0 = r0s[p], m = ms[p];
            double max_b = 0.0;
            if (jmode == ORC_J_HOST) {
                for (int j = 0; j < m; ++j)
                    for (int i = 0; i < n_sys; ++i) {
                        double v = fabs(AT(D, r0 + j, i));
                        if (v > max_b) max_b = v;
                    }
            } else {
                for (int i = 0; i < n_sys; ++i) {
                    double v0 = fabs(AT(D, r0, i)), vn = fabs(AT(D, r0 + m - 1, i));
                    if (v0 > max_b) max_b = v0;
                    if (vn > max_b) max_b = vn;
                }
            }
            double bound = (rhos[p] == 0.0 || rhos[p] >= 0.5) ? 0.0
                                                              : orc_rhs_bound_factor(rhos[p]) * max_b;
            int J = j_from_bound(rhos[p], bound, eps[p], m, jmode == ORC_J_DEVICE);
            /* The host solve clamps J to m-2 before use (filtered_tdma.cpp:224); the
             * device keeps J <= m-1 (its sweeps give the same x for J = m-1 and m-2)
             * and reports the unclamped value through last_J(). */
            Jrep[p] = J;
            if (J > m - 2) J = m - 2;
            if (jmode == ORC_J_HOST) Jrep[p] = J;
            Js[p] = J;
        }
    }

    /* Per segment: forward, backward, pack (filtered_tdma_kernels.hpp:35-189). */
    for (int p = 0; p < P; ++p) {
        int r0 = r0s[p], m = ms[p];
        int J = version == 2 ? Js[p] : m - 1; /* v1: full A update */
        int lo = version == 2 ? (m - 2) - J : -1;
        for (int i = 0; i < n_sys; ++i) {
#define S(arr, j) AT(arr, r0 + (j), i)
            double q0 = 1.0 / S(B, 0);
            S(A, 0) = S(A, 0) * q0;
            S(C, 0) = S(C, 0) * q0;
            S(D, 0) = S(D, 0) * q0;
            double q1 = 1.0 / S(B, 1);
            S(A, 1) = S(A, 1) * q1;
            S(C, 1) = S(C, 1) * q1;
            S(D, 1) = S(D, 1) * q1;
            for (int j = 2; j < m; ++j) {
                double a = S(A, j);
                double inv = 1.0 / (S(B, j) - a * S(C, j - 1));
                S(D, j) = inv * (S(D, j) - a * S(D, j - 1));
                S(C, j) = inv * S(C, j);
                if (j <= J) S(A, j) = -inv * a * S(A, j - 1);
            }
            for (int j = m - 3; j >= 1; --j) {
                double c = S(C, j);
                S(D, j) = S(D, j) - c * S(D, j + 1);
                if (version == 1 || j < J) S(A, j) = S(A, j) - c * S(A, j + 1);
                if (version == 1 || j > lo) S(C, j) = c * -S(C, j + 1);
            }
            double r = 1.0 / (1.0 - S(A, 1) * S(C, 0));
            S(D, 0) = r * (S(D, 0) - S(C, 0) * S(D, 1));
            S(A, 0) = r * S(A, 0);
#undef S
        }
    }

    /* Interface 2x2 solves with the neighbours' pre-interface rows
     * (filtered_tdma_kernels.hpp:197-218).  Save the exchanged rows first:
     * every segment uses its neighbours' values from before the update. */
    double* C_last = (double*)malloc(sizeof(double) * (size_t)P * n_sys);
    double* D_last = (double*)malloc(sizeof(double) * (size_t)P * n_sys);
    double* A_first = (double*)malloc(sizeof(double) * (size_t)P * n_sys);
    double* D_first = (double*)malloc(sizeof(double) * (size_t)P * n_sys);
    for (int p = 0; p < P; ++p)
        for (int i = 0; i < n_sys; ++i) {
            int last = r0s[p] + ms[p] - 1;
            C_last[(size_t)p * n_sys + i] = AT(C, last, i);
            D_last[(size_t)p * n_sys + i] = AT(D, last, i);
            A_first[(size_t)p * n_sys + i] = AT(A, r0s[p], i);
            D_first[(size_t)p * n_sys + i] = AT(D, r0s[p], i);
        }
    for (int p = 0; p < P; ++p) {
        int left = p - 1, right = p + 1;
        if (cyclic) {
            left = (p - 1 + P) % P;
            right = (p + 1) % P;
        }
        int has_left = left >= 0, has_right = right < P;
        int first = r0s[p], last = r0s[p] + ms[p] - 1;
        for (int i = 0; i < n_sys; ++i) {
            if (has_left) {
                double a0 = AT(A, first, i);
                AT(D, first, i) = (AT(D, first, i) - a0 * D_last[(size_t)left * n_sys + i]) /
                                  (1.0 - C_last[(size_t)left * n_sys + i] * a0);
            }
            if (has_right) {
                double cn = AT(C, last, i);
                AT(D, last, i) = (AT(D, last, i) - cn * D_first[(size_t)right * n_sys + i]) /
                                 (1.0 - A_first[(size_t)right * n_sys + i] * cn);
            }
        }
    }
    free(C_last);
    free(D_last);
    free(A_first);
    free(D_first);

    /* v1: J after the interface solve, from the post-interface boundary rows. */
    if (version == 1) {
        for (int p = 0; p < P; ++p) {
            int first = r0s[p], last = r0s[p] + ms[p] - 1, m = ms[p];
            double m0 = 0.0, mn = 0.0;
            for (int i = 0; i < n_sys; ++i) {
                double v0 = fabs(AT(D, first, i)), vn = fabs(AT(D, last, i));
                if (v0 > m0) m0 = v0;
                if (vn > mn) mn = vn;
            }
            double rho = rhos[p], bound = 0.0;
            if (!(rho == 0.0 || rho >= 0.5)) {
                if (jmode == ORC_J_HOST) {
                    double q = q_of(rho);
                    bound = (m0 + mn) * q / (1.0 - q);
                } else {
                    bound = orc_rhs_bound_factor(rho) * (m0 > mn ? m0 : mn);
                }
            }
            Js[p] = j_from_bound(rho, bound, eps[p], m, jmode == ORC_J_DEVICE);
            Jrep[p] = Js[p];
        }
    }

    /* Truncated correction (filtered_tdma_kernels.hpp:227-250):
     * rows 1..left_end get -A_j x_0, rows right_beg..m-2 get -C_j x_{m-1}. */
    for (int p = 0; p < P; ++p) {
        int r0 = r0s[p], m = ms[p], J = Js[p];
        int left_end = J < m - 2 ? J : m - 2;
        int right_beg = (m - 1) - J;
        if (right_beg < 1) right_beg = 1;
        for (int i = 0; i < n_sys; ++i) {
            double x0 = AT(D, r0, i), xn = AT(D, r0 + m - 1, i);
            for (int j = 1; j <= left_end; ++j)
                AT(D, r0 + j, i) = AT(D, r0 + j, i) - AT(A, r0 + j, i) * x0;
            for (int j = right_beg; j < m - 1; ++j)
                AT(D, r0 + j, i) = AT(D, r0 + j, i) - AT(C, r0 + j, i) * xn;
        }
        if (J_out) J_out[p] = Jrep[p];
    }
    free(r0s);
    free(ms);
    free(Js);
    free(Jrep);
    free(rhos);
    free(eps);
    return 0;
}

/* Per-row bound max(|A_k/B_k|, |C_k/B_k|) from system `sys`'s column, the
 * reference's estimate (apps/heat_cpu/tdma_backend.cpp:33-44 with sys = 0;
 * libs/filtered_tdma/gpu/filtered_tdma_kernels.cuh:46-67). */
void orc_rho_rows(const double* A, const double* B, const double* C, int n_sys, int n_row,
                  int sys, double* rho_row) {
    for (int k = 0; k < n_row; ++k) {
        double b = AT(B, k, sys);
        double ra = b != 0.0 ? fabs(AT(A, k, sys) / b) : 0.0;
        double rc = b != 0.0 ? fabs(AT(C, k, sys) / b) : 0.0;
        rho_row[k] = ra > rc ? ra : rc;
    }
}

/* Per-row bound as the maximum over all systems (a conservative estimate for
 * batches whose systems differ). */
void orc_rho_rows_all(const double* A, const double* B, const double* C, int n_sys, int n_row,
                      double* rho_row) {
    for (int k = 0; k < n_row; ++k) {
        double m = 0.0;
        for (int i = 0; i < n_sys; ++i) {
            double b = AT(B, k, i);
            double ra = b != 0.0 ? fabs(AT(A, k, i) / b) : 0.0;
            double rc = b != 0.0 ? fabs(AT(C, k, i) / b) : 0.0;
            if (ra > m) m = ra;
            if (rc > m) m = rc;
        }
        rho_row[k] = m;
    }
}
