// Reduced interface system of PaScaL's segmented solve, solved in registers
// with warp shuffles (the in-GPU replacement of the reference's all-to-all of
// reduced rows followed by a serial Thomas on 2P rows,
// libs/pascal_tdma/cpu/pascal_tdma.cpp:185-210).
//
// Row notation for sub-segment p of one system:
//   first: l0 xL(p-1) + xF(p) + u0 xL(p) = r0
//   last:  l1 xF(p) + xL(p) + u1 xF(p+1) = r1
// One cyclic-reduction level eliminates the first-row unknowns and leaves
//   a xL(p-1) + xL(p) + c xL(p+1) = d,
// which parallel cyclic reduction solves in log2(nseg) shuffle steps; the
// first-row unknowns follow from the first rows.
#pragma once

#include "btdma_common.cuh"

namespace btdma {

// One PCR row update of  l x_{i-dl} + x_i + u x_{i+dl} = r  with its
// neighbours (m: row i-dl, p: row i+dl).
__device__ __forceinline__ void pcr_step(double& l, double& u, double& r, double lm, double um,
                                         double rm, double lp, double up, double rp) {
    const double ib = rcp_nr(1.0 - l * um - u * lp);
    const double nl = -l * lm * ib;
    const double nu = -u * up * ib;
    r = (r - l * rm - u * rp) * ib;
    l = nl;
    u = nu;
}

// One system's reduced system over a group of W = 2^ceil(log2 nseg) <= 32
// consecutive lanes (lane p of the group holds sub-segment p; lanes with
// act == false carry identity rows).  Every lane of the warp must call it.
// Periodic systems (CYCLIC) need nseg to be a power of two.
template <bool CYCLIC>
__device__ __forceinline__ void reduced_solve_shfl(double l0, double u0, double r0, double l1,
                                                   double u1, double r1, int p, int nseg, int W,
                                                   bool act, double& xf, double& xl) {
    // next sub-segment's first row (zero past the end unless periodic)
    const int pn = (CYCLIC && p == nseg - 1) ? 0 : p + 1;
    double l0n = __shfl_sync(0xffffffffu, l0, pn, W);
    double u0n = __shfl_sync(0xffffffffu, u0, pn, W);
    double r0n = __shfl_sync(0xffffffffu, r0, pn, W);
    if (!CYCLIC && p + 1 >= nseg) l0n = u0n = r0n = 0.0;
    double al_ = 0, cl_ = 0, dl_ = 0;
    {
        const double ib = rcp_nr(1.0 - l1 * u0 - u1 * l0n);
        al_ = -l1 * l0 * ib;
        cl_ = -u1 * u0n * ib;
        dl_ = (r1 - l1 * r0 - u1 * r0n) * ib;
    }
    if (!act) al_ = cl_ = dl_ = 0.0;
    if (CYCLIC && nseg == 1) {
        xl = dl_ * rcp_nr(1.0 + al_ + cl_);
    } else {
        bool solved = false;
        xl = 0.0;
        for (int dl = 1; dl < nseg; dl <<= 1) {
            int im = p - dl, ip = p + dl;
            if (CYCLIC) {
                im = im < 0 ? im + nseg : im;
                ip = ip >= nseg ? ip - nseg : ip;
            }
            double lm = __shfl_sync(0xffffffffu, al_, im & (W - 1), W);
            double um = __shfl_sync(0xffffffffu, cl_, im & (W - 1), W);
            double rm = __shfl_sync(0xffffffffu, dl_, im & (W - 1), W);
            double lp = __shfl_sync(0xffffffffu, al_, ip & (W - 1), W);
            double up = __shfl_sync(0xffffffffu, cl_, ip & (W - 1), W);
            double rp = __shfl_sync(0xffffffffu, dl_, ip & (W - 1), W);
            if (!CYCLIC) {
                if (im < 0) lm = um = rm = 0.0;
                if (ip >= nseg) lp = up = rp = 0.0;
            }
            if (CYCLIC && 2 * dl == nseg) {
                // p-dl and p+dl are the same row j: 2x2 system in x_p, x_j
                const double si = al_ + cl_, sj = lm + um;
                xl = (dl_ - si * rm) * rcp_nr(1.0 - si * sj);
                solved = true;
            } else {
                pcr_step(al_, cl_, dl_, lm, um, rm, lp, up, rp);
            }
        }
        if (!solved) xl = dl_;
    }
    // x_first(p) = r0 - l0 xL(p-1) - u0 xL(p)
    const int pm = (CYCLIC && p == 0) ? nseg - 1 : p - 1;
    double xlm = __shfl_sync(0xffffffffu, xl, pm & (W - 1), W);
    if (!CYCLIC && p == 0) xlm = 0.0;
    xf = r0 - l0 * xlm - u0 * xl;
}

// Filtered's reduced system (FilteredTDMA v2, libs/filtered_tdma/cpu/
// filtered_tdma.cpp:217-238 with filtered_tdma_kernels.hpp's steps) in the
// lanes of reduced_solve_shfl: the sub-segments are grouped into segments of R
// consecutive lanes (R a power of two; the reference's ranks of m = 16 R rows).
// Inside a segment the system is solved exactly, with the two couplings to
// the neighbouring segments as parameters: three right-hand sides, y0 (the
// rows' own), yl (the left neighbour's last unknown = 1) and yr (the right
// neighbour's first unknown = 1), so every unknown is y0 + lam yl + rho yr.
// Across segments Filtered's approximation: the far couplings (a segment's
// first unknown's response to its right neighbour, its last unknown's to its
// left neighbour, of order rho^m) are dropped, which leaves one 2 x 2 system
// per interface (solve_interfaces, filtered_tdma_kernels.hpp:172-196):
//   f_k = y0F_k + yl F_k l_{k-1},  l_{k-1} = y0L_{k-1} + yr L_{k-1} f_k.
// lam and rho of each segment then come from its interfaces (0 outside the
// batch unless CYCLIC).  The J-row truncation of the correction is not
// applied: every row is back-substituted with the full correction, which costs
// nothing extra here; the result stays within Filtered's eps of the exact one.
template <bool CYCLIC>
__device__ __forceinline__ void reduced_solve_filtered(double l0, double u0, double r0, double l1,
                                                       double u1, double r1, int p, int nseg,
                                                       int W, int R, bool act, double& xf,
                                                       double& xl) {
    const unsigned FULL = 0xffffffffu;
    const int t = p & (R - 1);     // lane in the segment
    const int k0 = p - t;          // first lane of the segment
    const double l0s = t == 0 ? 0.0 : l0;  // couplings inside the segment only
    const double u1s = t == R - 1 ? 0.0 : u1;
    // the three right-hand sides of the first / last rows
    double a0 = r0, a1 = r1;
    double b0 = t == 0 ? -l0 : 0.0, b1 = 0.0;
    double c0 = 0.0, c1 = t == R - 1 ? -u1 : 0.0;
    // cyclic reduction: the next sub-segment's first row (inside the segment)
    const int pn = (p + 1) & (W - 1);
    const double l0n = __shfl_sync(FULL, l0, pn, W), u0n = __shfl_sync(FULL, u0, pn, W);
    const double a0n = __shfl_sync(FULL, a0, pn, W), b0n = __shfl_sync(FULL, b0, pn, W);
    const double c0n = __shfl_sync(FULL, c0, pn, W);
    const double ib = rcp_nr(1.0 - l1 * u0 - u1s * l0n);
    double al = -l1 * l0s * ib, cl = -u1s * u0n * ib;
    double da = (a1 - l1 * a0 - u1s * a0n) * ib;
    double db = (b1 - l1 * b0 - u1s * b0n) * ib;
    double dc = (c1 - l1 * c0 - u1s * c0n) * ib;
    if (!act) al = cl = da = db = dc = 0.0;
    // parallel cyclic reduction inside the segment
    for (int dl = 1; dl < R; dl <<= 1) {
        const bool vm = t - dl >= 0, vp = t + dl < R;
        const int im = (p - dl) & (W - 1), ip = (p + dl) & (W - 1);
        double lm = __shfl_sync(FULL, al, im, W), um = __shfl_sync(FULL, cl, im, W);
        double lp = __shfl_sync(FULL, al, ip, W), up = __shfl_sync(FULL, cl, ip, W);
        double am = __shfl_sync(FULL, da, im, W), ap = __shfl_sync(FULL, da, ip, W);
        double bm = __shfl_sync(FULL, db, im, W), bp = __shfl_sync(FULL, db, ip, W);
        double cm = __shfl_sync(FULL, dc, im, W), cp = __shfl_sync(FULL, dc, ip, W);
        if (!vm) lm = um = am = bm = cm = 0.0;
        if (!vp) lp = up = ap = bp = cp = 0.0;
        const double ibl = rcp_nr(1.0 - al * um - cl * lp);
        da = (da - al * am - cl * ap) * ibl;
        db = (db - al * bm - cl * bp) * ibl;
        dc = (dc - al * cm - cl * cp) * ibl;
        const double nl = -al * lm * ibl;
        cl = -cl * up * ibl;
        al = nl;
    }
    // last unknowns (da, db, dc); first unknowns from the first rows
    const int pm = (p - 1) & (W - 1);
    double xam = __shfl_sync(FULL, da, pm, W), xbm = __shfl_sync(FULL, db, pm, W);
    double xcm = __shfl_sync(FULL, dc, pm, W);
    if (t == 0) xam = xbm = xcm = 0.0;
    const double fa = a0 - l0s * xam - u0 * da;
    const double fb = b0 - l0s * xbm - u0 * db;
    const double fc = c0 - l0s * xcm - u0 * dc;
    // interface 2 x 2 at each segment's first lane: f_k and l_{k-1}, with
    // the previous segment's last lane's y0 and yr
    const int pl = (k0 - 1) & (W - 1);
    const double yl0 = __shfl_sync(FULL, da, pl, W), ylr = __shfl_sync(FULL, dc, pl, W);
    const bool left = CYCLIC || k0 > 0;
    double f = fa, lam = 0.0;
    if (left) {
        f = (fa + fb * yl0) * rcp_nr(1.0 - fb * ylr);
        lam = yl0 + ylr * f;
    }
    // every lane: lam of its segment (from its first lane) and rho (the next
    // segment's first lane's f)
    const int kn = (k0 + R) & (W - 1);
    const double lk = __shfl_sync(FULL, lam, k0, W);
    double rk = __shfl_sync(FULL, f, kn, W);
    if (!CYCLIC && k0 + R >= nseg) rk = 0.0;
    xf = fa + lk * fb + rk * fc;
    xl = da + lk * db + rk * dc;
}

// The matrix steps of reduced_solve_shfl for one lane, written to lt[0 .. 5 +
// 3 * levels) (the lane table of a matrix shared by every system, see
// reduced_solve_rhs).  Every lane of the warp calls it with the same nseg
// <= 32; lanes with act == false carry identity rows.
template <bool CYCLIC>
__device__ __forceinline__ void reduced_lane_table(double l0, double u0, double l1, double u1,
                                                   int p, int nseg, int W, bool act,
                                                   double* lt) {
    const int pn = (CYCLIC && p == nseg - 1) ? 0 : p + 1;
    double l0n = __shfl_sync(0xffffffffu, l0, pn, W);
    double u0n = __shfl_sync(0xffffffffu, u0, pn, W);
    const bool next = CYCLIC || p + 1 < nseg;
    if (!next) l0n = u0n = 0.0;
    const double ib = rcp_nr(1.0 - l1 * u0 - u1 * l0n);
    double al = act ? -l1 * l0 * ib : 0.0;
    double cl = act ? -u1 * u0n * ib : 0.0;
    if (lt) {
        lt[0] = act ? ib : 0.0;
        lt[1] = act ? l1 : 0.0;
        lt[2] = act && next ? u1 : 0.0;
        lt[3] = act ? l0 : 0.0;
        lt[4] = act ? u0 : 0.0;
    }
    if (CYCLIC && nseg == 1) {
        if (lt) {
            lt[5] = lt[6] = 0.0;
            lt[7] = rcp_nr(1.0 + al + cl);
        }
        return;
    }
    int v = 0;
    for (int dl = 1; dl < nseg; dl <<= 1, ++v) {
        int im = p - dl, ip = p + dl;
        if (CYCLIC) {
            im = im < 0 ? im + nseg : im;
            ip = ip >= nseg ? ip - nseg : ip;
        }
        double lm = __shfl_sync(0xffffffffu, al, im & (W - 1), W);
        double um = __shfl_sync(0xffffffffu, cl, im & (W - 1), W);
        double lp = __shfl_sync(0xffffffffu, al, ip & (W - 1), W);
        double up = __shfl_sync(0xffffffffu, cl, ip & (W - 1), W);
        const bool vm = CYCLIC || im >= 0, vp = CYCLIC || ip < nseg;
        if (!vm) lm = um = 0.0;
        if (!vp) lp = up = 0.0;
        double* lv = lt ? lt + 5 + 3 * v : nullptr;
        if (CYCLIC && 2 * dl == nseg) {
            // the 2x2 closing step: x_p = (r_p - (l + u) r_j) / (1 - (l + u)(l_j + u_j))
            const double si = al + cl;
            if (lv) {
                lv[0] = si;
                lv[1] = 0.0;
                lv[2] = rcp_nr(1.0 - si * (lm + um));
            }
            return;
        }
        const double ibl = rcp_nr(1.0 - al * um - cl * lp);
        if (lv) {
            lv[0] = vm ? al : 0.0;
            lv[1] = vp ? cl : 0.0;
            lv[2] = ibl;
        }
        const double nl = -al * lm * ibl;
        cl = -cl * up * ibl;
        al = nl;
    }
}

// reduced_solve_shfl for a batch whose systems share one matrix: lt is this
// lane's table from reduced_lane_table (entry k at lt[k * ls]), so only the
// right-hand sides travel (two shuffles and three operations per level, no
// reciprocals).  The right-hand-side arithmetic is that of reduced_solve_shfl.
template <bool CYCLIC>
__device__ __forceinline__ void reduced_solve_rhs(double r0, double r1, int p, int nseg, int W,
                                                  const double* __restrict__ lt, int ls,
                                                  double& xf, double& xl) {
    const int pn = (CYCLIC && p == nseg - 1) ? 0 : p + 1;
    const double r0n = __shfl_sync(0xffffffffu, r0, pn & (W - 1), W);
    double r = (r1 - lt[1 * ls] * r0 - lt[2 * ls] * r0n) * lt[0 * ls];
    if (CYCLIC && nseg == 1) {
        r *= lt[7 * ls];
    } else {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const int dl = 1 << v;
            if (dl >= nseg) break;
            int im = p - dl, ip = p + dl;
            if (CYCLIC) {
                im = im < 0 ? im + nseg : im;
                ip = ip >= nseg ? ip - nseg : ip;
            }
            const double rm = __shfl_sync(0xffffffffu, r, im & (W - 1), W);
            const double rp = __shfl_sync(0xffffffffu, r, ip & (W - 1), W);
            r = (r - lt[(5 + 3 * v) * ls] * rm - lt[(6 + 3 * v) * ls] * rp) * lt[(7 + 3 * v) * ls];
            if (CYCLIC && 2 * dl == nseg) break;
        }
    }
    xl = r;
    const int pm = (CYCLIC && p == 0) ? nseg - 1 : p - 1;
    double xlm = __shfl_sync(0xffffffffu, xl, pm & (W - 1), W);
    if (!CYCLIC && p == 0) xlm = 0.0;
    xf = r0 - lt[3 * ls] * xlm - lt[4 * ls] * xl;
}

}  // namespace btdma
