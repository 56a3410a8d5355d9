// Common device helpers for the batched tridiagonal kernels (sm_100a only).
//
// * exact FP64/FP32 arithmetic wrappers: the kernels that promise bit-identical
//   results to the reference's CPU code (which is compiled without fused
//   multiply-add) use round-to-nearest intrinsics, which the compiler never
//   contracts into FMA;
// * mbarrier / TMA (cp.async.bulk.tensor) wrappers written in inline PTX, no
//   multicast anywhere;
// * the device status word: kernels never trap; they OR a bit into a status
//   word that the host reads with btdma_status().
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "btdma.h"

#ifndef __CUDA_ARCH__
#define BTDMA_HOST_ONLY 1
#endif

namespace btdma {

// ---------------------------------------------------------------- arithmetic
struct Exact64 {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double rcp(double a) { return __drcp_rn(a); }
};

// Reciprocal for the kernels that promise rounding-level accuracy, not bit
// identity: the hardware approximation rcp.approx.ftz.f64 refined by two
// Newton-Raphson steps e = 1 - x r, r += r e (each step squares the relative
// error), with no special-case branches.  Accurate to about an ulp for normal,
// finite, non-zero x; zero, infinite or subnormal pivots are not handled (they
// are not valid inputs of a diagonally dominant system).
__device__ __forceinline__ double rcp_nr(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

// Status bits OR-ed into the device status word.
enum : unsigned {
    ST_TIMEOUT = 1u << 0,     // an mbarrier wait hit its iteration limit
    ST_NONFINITE = 1u << 1,   // a solution entry is NaN or Inf
};

__device__ __forceinline__ void raise_status(unsigned* status, unsigned bit) {
    if (status) atomicOr(status, bit);
}

// ------------------------------------------------------------------ mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// One poll.  The thread may be suspended until the phase completes or for at
// most ~kSuspendNs, so a waiting warp sleeps instead of spinning.
constexpr uint32_t kSuspendNs = 20000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each poll suspends the thread for
// at most kSuspendNs), raising ST_TIMEOUT.  Every 64 polls it also checks the
// status word and gives up at once if another CTA already timed out, so a
// systematic failure costs one timeout, not one per CTA.
static __device__ __noinline__ bool mbar_wait_slow(uint64_t* bar, uint32_t parity, unsigned* status,
                                            uint32_t limit);

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  unsigned* status, uint32_t limit = 1u << 16) {
    // fast path: one poll (it suspends until the phase completes or briefly times out)
    if (mbar_try_wait(bar, parity)) return true;
    return mbar_wait_slow(bar, parity, status, limit);
}

// One poll without a suspend-time hint: the hardware's own, shorter limit, so a
// waiting warp polls again sooner.  Measured faster than the hinted poll for the
// wide tiled kernel (every warp waits on every stage) and slower for the narrow
// one.
__device__ __forceinline__ bool mbar_try_wait_spin(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

static __device__ __noinline__ bool mbar_wait_spin_slow(uint64_t* bar, uint32_t parity,
                                                        unsigned* status, uint32_t limit) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (mbar_try_wait_spin(bar, parity)) return true;
        if (status && (it & 1023u) == 1023u &&
            (*reinterpret_cast<volatile unsigned*>(status) & ST_TIMEOUT))
            return false;
    }
    raise_status(status, ST_TIMEOUT);
    return false;
}

// Bounded wait with unhinted polls (a poll lasts far less than kSuspendNs, so
// the default limit allows more of them).
__device__ __forceinline__ bool mbar_wait_bounded_spin(uint64_t* bar, uint32_t parity,
                                                       unsigned* status,
                                                       uint32_t limit = 1u << 22) {
    if (mbar_try_wait_spin(bar, parity)) return true;
    return mbar_wait_spin_slow(bar, parity, status, limit);
}

static __device__ __noinline__ bool mbar_wait_slow(uint64_t* bar, uint32_t parity, unsigned* status,
                                            uint32_t limit) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (status && (it & 63u) == 63u &&
            (*reinterpret_cast<volatile unsigned*>(status) & ST_TIMEOUT))
            return false;
    }
    raise_status(status, ST_TIMEOUT);
    return false;
}

// ------------------------------------------------------------------------ TMA
// 2-D tiled load global -> this CTA's shared memory, completion on `bar`.
// x = innermost coordinate (system index, a multiple of the tile width, so its
// byte offset is a multiple of 16), y = row.
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// 2-D tiled store shared -> global (bulk group).  Out-of-range elements of the
// box are not written.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y,
                                             const void* smem_src) {
    asm volatile(
        "cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(x), "r"(y), "r"(smem_u32(smem_src))
        : "memory");
}

__device__ __forceinline__ void tma_store_commit() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__device__ __forceinline__ void tma_store_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

__device__ __forceinline__ void tma_store_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Make generic-proxy writes to shared memory visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ------------------------------------------------------------- segmentation
// Block split of n rows into P segments (first `rem` segments one row longer),
// the reference's para_range (libs/pascal_tdma/cpu/para_range.cpp:4-10).
__host__ __device__ __forceinline__ void seg_range(int n, int P, int k, int& r0, int& m) {
    int base = n / P, rem = n % P;
    r0 = k * base + (k < rem ? k : rem);
    m = base + (k < rem ? 1 : 0);
}

}  // namespace btdma
