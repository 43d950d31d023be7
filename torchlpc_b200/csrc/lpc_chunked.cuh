// Chunked linear-recurrence scan kernels (parallel in time).
#pragma once

#include "lpc_plain.cuh"

namespace lpcb {

// Largest filter order any entry point accepts (the reference's limit,
// torchlpc/csrc/cuda/lpc.cu:135).
constexpr int64_t kMaxOrder = 1024;

bool chunked_supported(int64_t N);
// Process-wide error word the chunked kernels OR a nonzero status into.
void set_error_word(unsigned *word);
// Target chunk length of the chunked scan (process-wide; <= 0 restores the
// default, chosen by signal length; chunk_target() then returns 0); the plan
// rounds it to an even number of windows.
void set_chunk_target(int64_t samples);
int64_t chunk_target();
bool chunked_preferred(int64_t B, int64_t T, int64_t N, int64_t a_stride_t);
size_t chunked_forward_workspace(size_t esz, int64_t B, int64_t T, int64_t N, int64_t a_stride_t);
size_t chunked_backward_workspace(size_t esz, int64_t B, int64_t T, int64_t N, int64_t a_stride_t);

// Ragged batches (signals concatenated along time, int64 offsets on the device).
size_t chunked_ragged_workspace(size_t esz, int64_t nsig, int64_t S, int64_t N);
template <typename T>
cudaError_t chunked_forward_ragged(const T *x, const T *A, const int64_t *off, const T *zi, T *y, int64_t nsig,
                                   int64_t S, int64_t N, void *ws, size_t ws_bytes, cudaStream_t st);
template <typename T>
cudaError_t chunked_backward_ragged(const T *gy, const T *A, const int64_t *off, const T *zi, const T *y, T *gx,
                                    T *gA, T *gzi, int64_t nsig, int64_t S, int64_t N, void *ws, size_t ws_bytes,
                                    cudaStream_t st);

// Boundary-state checkpointing (time-varying coefficients): the forward keeps
// every chunk's entry state, the backward recomputes y from them and x.
int64_t chunked_checkpoint_chunk(size_t esz, int64_t T, int64_t N);
int64_t chunked_checkpoint_elems(size_t esz, int64_t B, int64_t T, int64_t N, int64_t chunk);
size_t chunked_forward_ckpt_workspace(size_t esz, int64_t B, int64_t T, int64_t N, int64_t chunk);
size_t chunked_backward_ckpt_workspace(size_t esz, int64_t B, int64_t T, int64_t N, int64_t chunk);
template <typename T>
cudaError_t chunked_forward_ckpt(const FwdArgs<T> &a, T *states, int64_t chunk, void *ws, size_t ws_bytes,
                                 cudaStream_t st);
template <typename T>
cudaError_t chunked_backward_ckpt(const BwdArgs<T> &a, const T *x, const T *states, int64_t chunk, void *ws,
                                  size_t ws_bytes, cudaStream_t st);

// Failure detection: a launch whose look-back wait runs out (no GPU fault).
size_t chunked_selftest_workspace();
cudaError_t chunked_selftest_timeout(void *ws, size_t ws_bytes, unsigned spin_limit, cudaStream_t st);

template <typename T>
cudaError_t chunked_forward(const FwdArgs<T> &p, bool neg, void *ws, size_t ws_bytes,
                            cudaStream_t st);
template <typename T>
cudaError_t chunked_backward(const BwdArgs<T> &p, bool neg, void *ws, size_t ws_bytes,
                             cudaStream_t st);

}  // namespace lpcb
