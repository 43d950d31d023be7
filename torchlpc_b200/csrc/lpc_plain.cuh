// Argument blocks and entry points of the plain (sequential) kernels.
#pragma once

#include "lpc_common.cuh"

namespace lpcb {

template <typename F>
struct FwdArgs {
    const F *x;     // (B,T) dense
    const F *A;     // A[b,t,i] = A[b*a_stride_b + t*a_stride_t + i]
    const F *zi;    // (B,N) or nullptr
    F *y;           // (B,T) dense
    int64_t B, T, N, a_stride_b, a_stride_t;
};

template <typename F>
struct BwdArgs {
    const F *gy;    // (B,T)
    const F *A;
    const F *zi;    // (B,N) or nullptr
    const F *y;     // (B,T) forward output
    F *gx;          // (B,T)
    F *gA;          // (B,T,N) dense, (B,N) when a_stride_t == 0, or nullptr
    F *gzi;         // (B,N) or nullptr
    int64_t B, T, N, a_stride_b, a_stride_t;
};

// neg: the stored coefficients are the negated filter taps (order-1 scan,
// out[t] = decay[t]*out[t-1] + impulse[t]  <=>  A = -decay); the coefficient
// gradient is then taken with respect to the stored values.
template <typename T>
cudaError_t plain_forward(const FwdArgs<T> &p, bool neg, cudaStream_t st);
template <typename T>
cudaError_t plain_backward(const BwdArgs<T> &p, bool neg, cudaStream_t st);

}  // namespace lpcb
