// Time-invariant all-pole filter (one coefficient set per signal).
#pragma once

#include "lpc_plain.cuh"

namespace lpcb {

bool ti_supported(int64_t N);
size_t ti_workspace(size_t esz, int64_t B, int64_t T, int64_t N);

// Filters for a_stride_t == 0 (coefficients a[b,i] = A[b*a_stride_b + i]).
template <typename T>
cudaError_t ti_forward(const FwdArgs<T> &p, void *ws, size_t ws_bytes, cudaStream_t st);
template <typename T>
cudaError_t ti_backward(const BwdArgs<T> &p, void *ws, size_t ws_bytes, cudaStream_t st);

// grad_a[b,i] = sgn * sum_t grad_x[b,t] * y[b,t-1-i] (y[b,-1-k] = zi[b,k]),
// sgn = -1 (or +1 for negated stored coefficients); overwrites ga (B,N).
template <typename T>
cudaError_t ti_grad_a(const T *gx, const T *y, const T *zi, T *ga, int64_t B, int64_t T_, int64_t N, bool neg,
                      cudaStream_t st);

}  // namespace lpcb
