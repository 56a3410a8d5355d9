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
