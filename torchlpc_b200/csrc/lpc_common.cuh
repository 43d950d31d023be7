// Shared device helpers for the lpc_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lpc_b200.h"

namespace lpcb {

// Padded orders that get a register-resident history (fully unrolled ring).
// An order N runs on the smallest padded order NP >= N; padded taps carry
// zero coefficients.  Orders above 32 use the warp-split kernels.
#define LPCB_FOR_EACH_NP(X) X(1) X(2) X(4) X(8) X(12) X(16) X(20) X(24) X(28) X(32)

__host__ __device__ __forceinline__ int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int64_t max64(int64_t a, int64_t b) { return a > b ? a : b; }

inline int padded_order(int64_t N) {
    if (N <= 1) return 1;
    if (N <= 2) return 2;
    if (N <= 4) return 4;
    if (N <= 8) return 8;
    if (N <= 12) return 12;
    if (N <= 16) return 16;
    if (N <= 20) return 20;
    if (N <= 24) return 24;
    if (N <= 28) return 28;
    if (N <= 32) return 32;
    return 0;  // warp-split kernels
}

// Batch of time steps staged per round trip: a multiple of NP near 64.
__host__ __device__ constexpr int plain_rows(int NP) { return NP * ((64 + NP - 1) / NP); }

__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
    static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async size");
    if constexpr (BYTES == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem)), "l"(gmem)
                     : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_addr(smem)), "l"(gmem),
                     "n"(BYTES)
                     : "memory");
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

template <typename T>
__device__ __forceinline__ T fmadd(T a, T b, T c) {
    return fma(a, b, c);
}

// Copy `count` elements of a row from global to shared, 16-byte vectors when
// both sides are aligned, element-wise otherwise.  Called by all lanes of a
// warp with the same arguments; lane `lane` takes every 32nd piece.
template <typename T>
__device__ __forceinline__ void warp_copy_row_async(T *dst, const T *src, int count, int lane,
                                                    bool vec_ok) {
    constexpr int V = 16 / sizeof(T);
    if (vec_ok) {
        for (int v = lane; v < count / V; v += 32) cp_async<16>(dst + v * V, src + v * V);
    } else {
        for (int e = lane; e < count; e += 32) cp_async<sizeof(T)>(dst + e, src + e);
    }
}

}  // namespace lpcb
