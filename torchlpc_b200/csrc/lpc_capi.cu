// extern "C" entry points of liblpc_b200 (declared in include/lpc_b200.h).
//
// Each entry point validates its arguments, picks the kernel family and
// launches asynchronously on the caller's stream.  Nothing here allocates.
#include <cstring>

#include "lpc_chunked.cuh"
#include "lpc_plain.cuh"
#include "lpc_ti.cuh"

using namespace lpcb;

namespace {

int cuda_status(cudaError_t e) { return e == cudaSuccess ? LPC_OK : LPC_ERR_CUDA; }

bool dtype_ok(int dtype) { return dtype == LPC_F32 || dtype == LPC_F64; }

bool sizes_ok(int64_t B, int64_t T, int64_t N) {
    return B >= 0 && T >= 0 && N >= 1 && N <= kMaxOrder && B < (int64_t(1) << 31);
}

// Choice between the sequential, the chunked and the time-invariant kernels.
// LPC_ALGO_CHUNKED falls back to the plain kernels for orders the chunked
// kernels do not cover (N > 32); LPC_ALGO_TI applies to a_stride_t == 0 only.
// AUTO: time-invariant coefficients with at least 2048 samples per signal take
// the time-invariant scan, long time-varying signals the chunked scan.
int resolve_algo(int algo, int64_t B, int64_t T, int64_t N, int64_t a_stride_t) {
    if (algo == LPC_ALGO_PLAIN) return algo;
    if (algo == LPC_ALGO_CHUNKED) return chunked_supported(N) ? algo : LPC_ALGO_PLAIN;
    if (a_stride_t == 0 && ti_supported(N) && (algo == LPC_ALGO_TI || T >= 2048)) return LPC_ALGO_TI;
    return chunked_preferred(B, T, N, a_stride_t) ? LPC_ALGO_CHUNKED : LPC_ALGO_PLAIN;
}

size_t workspace_for(int algo, size_t esz, int64_t B, int64_t T, int64_t N, int64_t a_stride_t) {
    if (algo == LPC_ALGO_CHUNKED) return chunked_forward_workspace(esz, B, T, N, a_stride_t);
    if (algo == LPC_ALGO_TI) return ti_workspace(esz, B, T, N);
    return 0;
}

template <typename T>
int forward_t(int algo, const void *x, const void *A, const void *zi, void *y, int64_t B,
              int64_t T_, int64_t N, int64_t sb, int64_t st, void *ws, size_t ws_bytes,
              cudaStream_t stream) {
    FwdArgs<T> p{static_cast<const T *>(x), static_cast<const T *>(A), static_cast<const T *>(zi),
                 static_cast<T *>(y), B, T_, N, sb, st};
    if (B == 0 || T_ == 0) return LPC_OK;
    if (algo == LPC_ALGO_CHUNKED) {
        if (ws_bytes < chunked_forward_workspace(sizeof(T), B, T_, N, st)) return LPC_ERR_WORKSPACE;
        return cuda_status(chunked_forward<T>(p, false, ws, ws_bytes, stream));
    }
    if (algo == LPC_ALGO_TI) {
        if (!ws || ws_bytes < ti_workspace(sizeof(T), B, T_, N)) return LPC_ERR_WORKSPACE;
        return cuda_status(ti_forward<T>(p, ws, ws_bytes, stream));
    }
    return cuda_status(plain_forward<T>(p, false, stream));
}

template <typename T>
int backward_t(int algo, const void *gy, const void *A, const void *zi, const void *y, void *gx,
               void *gA, void *gzi, int64_t B, int64_t T_, int64_t N, int64_t sb, int64_t st,
               void *ws, size_t ws_bytes, cudaStream_t stream) {
    BwdArgs<T> p{static_cast<const T *>(gy), static_cast<const T *>(A), static_cast<const T *>(zi),
                 static_cast<const T *>(y), static_cast<T *>(gx), static_cast<T *>(gA),
                 static_cast<T *>(gzi), B, T_, N, sb, st};
    if (B == 0) return LPC_OK;
    if (T_ == 0) {  // no samples: every gradient is zero
        if (gA && st == 0) cudaMemsetAsync(gA, 0, (size_t)B * N * sizeof(T), stream);
        if (gzi) cudaMemsetAsync(gzi, 0, (size_t)B * N * sizeof(T), stream);
        return cuda_status(cudaGetLastError());
    }
    if (algo == LPC_ALGO_CHUNKED) {
        if (ws_bytes < chunked_backward_workspace(sizeof(T), B, T_, N, st)) return LPC_ERR_WORKSPACE;
        return cuda_status(chunked_backward<T>(p, false, ws, ws_bytes, stream));
    }
    if (algo == LPC_ALGO_TI) {
        if (!ws || ws_bytes < ti_workspace(sizeof(T), B, T_, N)) return LPC_ERR_WORKSPACE;
        return cuda_status(ti_backward<T>(p, ws, ws_bytes, stream));
    }
    return cuda_status(plain_backward<T>(p, false, stream));
}

}  // namespace

extern "C" {

const char *lpc_b200_status_string(int status) {
    switch (status) {
        case LPC_OK: return "ok";
        case LPC_ERR_INVALID_ARGUMENT: return "invalid argument";
        case LPC_ERR_UNSUPPORTED: return "unsupported configuration";
        case LPC_ERR_WORKSPACE: return "workspace missing or too small";
        case LPC_ERR_CUDA: return "CUDA runtime error";
        case LPC_ERR_TIMEOUT: return "bounded device-side wait timed out";
        default: return "unknown status";
    }
}

int lpc_b200_version(void) { return 100; }

int lpc_b200_set_chunk_length(int64_t samples) {
    set_chunk_target(samples);
    return LPC_OK;
}

int64_t lpc_b200_chunk_length(void) { return chunk_target(); }

size_t lpc_b200_forward_workspace_size(int dtype, int algo, int64_t B, int64_t T, int64_t N,
                                       int64_t a_stride_t) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, N)) return 0;
    return workspace_for(resolve_algo(algo, B, T, N, a_stride_t), dtype == LPC_F32 ? 4 : 8, B, T, N, a_stride_t);
}

int lpc_b200_forward(int dtype, int algo, const void *x, const void *A, const void *zi, void *y,
                     int64_t B, int64_t T, int64_t N, int64_t a_stride_b, int64_t a_stride_t,
                     void *workspace, size_t workspace_bytes, void *stream) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, N)) return LPC_ERR_INVALID_ARGUMENT;
    if (B > 0 && T > 0 && (!x || !A || !y)) return LPC_ERR_INVALID_ARGUMENT;
    if (a_stride_t < 0 || a_stride_b < 0 || (a_stride_t != 0 && a_stride_t < N))
        return LPC_ERR_INVALID_ARGUMENT;
    algo = resolve_algo(algo, B, T, N, a_stride_t);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == LPC_F32)
        return forward_t<float>(algo, x, A, zi, y, B, T, N, a_stride_b, a_stride_t, workspace,
                                workspace_bytes, s);
    return forward_t<double>(algo, x, A, zi, y, B, T, N, a_stride_b, a_stride_t, workspace,
                             workspace_bytes, s);
}

size_t lpc_b200_backward_workspace_size(int dtype, int algo, int64_t B, int64_t T, int64_t N,
                                        int64_t a_stride_t) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, N)) return 0;
    return workspace_for(resolve_algo(algo, B, T, N, a_stride_t), dtype == LPC_F32 ? 4 : 8, B, T, N, a_stride_t);
}

int lpc_b200_backward(int dtype, int algo, const void *grad_y, const void *A, const void *zi,
                      const void *y, void *grad_x, void *grad_A, void *grad_zi, int64_t B,
                      int64_t T, int64_t N, int64_t a_stride_b, int64_t a_stride_t,
                      void *workspace, size_t workspace_bytes, void *stream) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, N)) return LPC_ERR_INVALID_ARGUMENT;
    if (B > 0 && T > 0 && (!grad_y || !A || !y || !grad_x)) return LPC_ERR_INVALID_ARGUMENT;
    if (a_stride_t < 0 || a_stride_b < 0 || (a_stride_t != 0 && a_stride_t < N))
        return LPC_ERR_INVALID_ARGUMENT;
    algo = resolve_algo(algo, B, T, N, a_stride_t);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == LPC_F32)
        return backward_t<float>(algo, grad_y, A, zi, y, grad_x, grad_A, grad_zi, B, T, N,
                                 a_stride_b, a_stride_t, workspace, workspace_bytes, s);
    return backward_t<double>(algo, grad_y, A, zi, y, grad_x, grad_A, grad_zi, B, T, N,
                              a_stride_b, a_stride_t, workspace, workspace_bytes, s);
}

int64_t lpc_b200_checkpoint_chunk(int dtype, int64_t T, int64_t N) {
    if (!dtype_ok(dtype) || !sizes_ok(1, T, N) || !chunked_supported(N)) return 0;
    return chunked_checkpoint_chunk(dtype == LPC_F32 ? 4 : 8, T, N);
}

int64_t lpc_b200_checkpoint_elems(int dtype, int64_t B, int64_t T, int64_t N, int64_t chunk_len) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, N)) return 0;
    return chunked_checkpoint_elems(dtype == LPC_F32 ? 4 : 8, B, T, N, chunk_len);
}

size_t lpc_b200_forward_checkpointed_workspace_size(int dtype, int64_t B, int64_t T, int64_t N,
                                                    int64_t chunk_len) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, N)) return 0;
    return chunked_forward_ckpt_workspace(dtype == LPC_F32 ? 4 : 8, B, T, N, chunk_len);
}

size_t lpc_b200_backward_checkpointed_workspace_size(int dtype, int64_t B, int64_t T, int64_t N,
                                                     int64_t chunk_len) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, N)) return 0;
    return chunked_backward_ckpt_workspace(dtype == LPC_F32 ? 4 : 8, B, T, N, chunk_len);
}

namespace {
int ckpt_check(int dtype, int64_t B, int64_t T, int64_t N, int64_t sb, int64_t st, int64_t chunk_len) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, N) || chunk_len <= 0) return LPC_ERR_INVALID_ARGUMENT;
    if (st < N || sb < 0) return st == 0 ? LPC_ERR_UNSUPPORTED : LPC_ERR_INVALID_ARGUMENT;
    if (!chunked_supported(N)) return LPC_ERR_UNSUPPORTED;
    return LPC_OK;
}
}  // namespace

int lpc_b200_forward_checkpointed(int dtype, const void *x, const void *A, const void *zi, void *y,
                                  void *states, int64_t B, int64_t T, int64_t N, int64_t a_stride_b,
                                  int64_t a_stride_t, int64_t chunk_len, void *workspace,
                                  size_t workspace_bytes, void *stream) {
    const int rc = ckpt_check(dtype, B, T, N, a_stride_b, a_stride_t, chunk_len);
    if (rc != LPC_OK) return rc;
    if (B == 0 || T == 0) return LPC_OK;
    if (!x || !A || !y || !states) return LPC_ERR_INVALID_ARGUMENT;
    const size_t esz = dtype == LPC_F32 ? 4 : 8;
    if (!workspace || workspace_bytes < chunked_forward_ckpt_workspace(esz, B, T, N, chunk_len))
        return LPC_ERR_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto run = [&](auto tag) -> int {
        using Tt = decltype(tag);
        FwdArgs<Tt> p{static_cast<const Tt *>(x), static_cast<const Tt *>(A), static_cast<const Tt *>(zi),
                      static_cast<Tt *>(y), B, T, N, a_stride_b, a_stride_t};
        return cuda_status(chunked_forward_ckpt<Tt>(p, static_cast<Tt *>(states), chunk_len, workspace,
                                                    workspace_bytes, s));
    };
    return dtype == LPC_F32 ? run(float{}) : run(double{});
}

int lpc_b200_backward_checkpointed(int dtype, const void *grad_y, const void *A, const void *zi,
                                   const void *x, const void *states, void *grad_x, void *grad_A,
                                   void *grad_zi, int64_t B, int64_t T, int64_t N, int64_t a_stride_b,
                                   int64_t a_stride_t, int64_t chunk_len, void *workspace,
                                   size_t workspace_bytes, void *stream) {
    const int rc = ckpt_check(dtype, B, T, N, a_stride_b, a_stride_t, chunk_len);
    if (rc != LPC_OK) return rc;
    if (B == 0) return LPC_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t esz = dtype == LPC_F32 ? 4 : 8;
    if (T == 0) {
        if (grad_zi) cudaMemsetAsync(grad_zi, 0, (size_t)B * N * esz, s);
        return cuda_status(cudaGetLastError());
    }
    if (!grad_y || !A || !x || !states || !grad_x) return LPC_ERR_INVALID_ARGUMENT;
    if (!workspace || workspace_bytes < chunked_backward_ckpt_workspace(esz, B, T, N, chunk_len))
        return LPC_ERR_WORKSPACE;
    auto run = [&](auto tag) -> int {
        using Tt = decltype(tag);
        BwdArgs<Tt> p{static_cast<const Tt *>(grad_y), static_cast<const Tt *>(A), static_cast<const Tt *>(zi),
                      nullptr, static_cast<Tt *>(grad_x), static_cast<Tt *>(grad_A),
                      static_cast<Tt *>(grad_zi), B, T, N, a_stride_b, a_stride_t};
        return cuda_status(chunked_backward_ckpt<Tt>(p, static_cast<const Tt *>(x),
                                                     static_cast<const Tt *>(states), chunk_len, workspace,
                                                     workspace_bytes, s));
    };
    return dtype == LPC_F32 ? run(float{}) : run(double{});
}

int lpc_b200_workspace_status(const void *workspace, unsigned *status, void *stream) {
    if (!workspace || !status) return LPC_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the status word follows the ticket counter in the workspace header
    if (cudaMemcpyAsync(status, static_cast<const unsigned char *>(workspace) + sizeof(unsigned), sizeof(unsigned),
                        cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return LPC_ERR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? LPC_OK : LPC_ERR_CUDA;
}

int lpc_b200_set_error_word(unsigned *word) {
    set_error_word(word);
    return LPC_OK;
}

size_t lpc_b200_selftest_workspace_size(void) { return chunked_selftest_workspace(); }

int lpc_b200_selftest_timeout(void *workspace, size_t workspace_bytes, unsigned spin_limit, unsigned *status,
                              void *stream) {
    if (!workspace || !status || spin_limit == 0) return LPC_ERR_INVALID_ARGUMENT;
    if (workspace_bytes < chunked_selftest_workspace()) return LPC_ERR_WORKSPACE;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (chunked_selftest_timeout(workspace, workspace_bytes, spin_limit, s) != cudaSuccess) return LPC_ERR_CUDA;
    const int rc = lpc_b200_workspace_status(workspace, status, stream);
    if (rc != LPC_OK) return rc;
    return *status != 0u ? LPC_ERR_TIMEOUT : LPC_OK;
}

size_t lpc_b200_ragged_workspace_size(int dtype, int64_t nsig, int64_t S, int64_t N) {
    if (!dtype_ok(dtype) || nsig < 0 || S < 0 || N < 1 || N > kMaxOrder) return 0;
    if (!chunked_supported(N) || nsig == 0) return 0;
    return chunked_ragged_workspace(dtype == LPC_F32 ? 4 : 8, nsig, S, N);
}

namespace {
int ragged_check(int dtype, const int64_t *offsets, int64_t nsig, int64_t S, int64_t N, void *ws,
                 size_t wsb) {
    if (!dtype_ok(dtype) || nsig < 0 || S < 0 || N < 1 || N > kMaxOrder || nsig >= (int64_t(1) << 31))
        return LPC_ERR_INVALID_ARGUMENT;
    if (nsig > 0 && !offsets) return LPC_ERR_INVALID_ARGUMENT;
    if (!chunked_supported(N)) return LPC_ERR_UNSUPPORTED;
    if (nsig > 0 && (!ws || wsb < chunked_ragged_workspace(dtype == LPC_F32 ? 4 : 8, nsig, S, N)))
        return LPC_ERR_WORKSPACE;
    return LPC_OK;
}
}  // namespace

int lpc_b200_forward_ragged(int dtype, const void *x, const void *A, const int64_t *offsets,
                            const void *zi, void *y, int64_t nsig, int64_t S, int64_t N,
                            void *workspace, size_t workspace_bytes, void *stream) {
    const int rc = ragged_check(dtype, offsets, nsig, S, N, workspace, workspace_bytes);
    if (rc != LPC_OK) return rc;
    if (nsig == 0) return LPC_OK;
    if (S > 0 && (!x || !A || !y)) return LPC_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == LPC_F32)
        return cuda_status(chunked_forward_ragged<float>(
            static_cast<const float *>(x), static_cast<const float *>(A), offsets,
            static_cast<const float *>(zi), static_cast<float *>(y), nsig, S, N, workspace,
            workspace_bytes, s));
    return cuda_status(chunked_forward_ragged<double>(
        static_cast<const double *>(x), static_cast<const double *>(A), offsets,
        static_cast<const double *>(zi), static_cast<double *>(y), nsig, S, N, workspace,
        workspace_bytes, s));
}

int lpc_b200_backward_ragged(int dtype, const void *grad_y, const void *A, const int64_t *offsets,
                             const void *zi, const void *y, void *grad_x, void *grad_A,
                             void *grad_zi, int64_t nsig, int64_t S, int64_t N, void *workspace,
                             size_t workspace_bytes, void *stream) {
    const int rc = ragged_check(dtype, offsets, nsig, S, N, workspace, workspace_bytes);
    if (rc != LPC_OK) return rc;
    if (nsig == 0) return LPC_OK;
    if (S > 0 && (!grad_y || !A || !y || !grad_x)) return LPC_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == LPC_F32)
        return cuda_status(chunked_backward_ragged<float>(
            static_cast<const float *>(grad_y), static_cast<const float *>(A), offsets,
            static_cast<const float *>(zi), static_cast<const float *>(y),
            static_cast<float *>(grad_x), static_cast<float *>(grad_A), static_cast<float *>(grad_zi),
            nsig, S, N, workspace, workspace_bytes, s));
    return cuda_status(chunked_backward_ragged<double>(
        static_cast<const double *>(grad_y), static_cast<const double *>(A), offsets,
        static_cast<const double *>(zi), static_cast<const double *>(y),
        static_cast<double *>(grad_x), static_cast<double *>(grad_A), static_cast<double *>(grad_zi),
        nsig, S, N, workspace, workspace_bytes, s));
}

size_t lpc_b200_scan_workspace_size(int dtype, int algo, int64_t B, int64_t T) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, 1)) return 0;
    if (resolve_algo(algo, B, T, 1, 1) != LPC_ALGO_CHUNKED) return 0;
    return chunked_forward_workspace(dtype == LPC_F32 ? 4 : 8, B, T, 1, 1);
}

int lpc_b200_scan(int dtype, int algo, const void *impulse, const void *decay, const void *init,
                  void *out, int64_t B, int64_t T, void *workspace, size_t workspace_bytes,
                  void *stream) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, 1)) return LPC_ERR_INVALID_ARGUMENT;
    if (B > 0 && T > 0 && (!impulse || !decay || !out)) return LPC_ERR_INVALID_ARGUMENT;
    if (B == 0 || T == 0) return LPC_OK;
    algo = resolve_algo(algo, B, T, 1, 1);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto run = [&](auto tag) -> int {
        using Tt = decltype(tag);
        FwdArgs<Tt> p{static_cast<const Tt *>(impulse), static_cast<const Tt *>(decay),
                      static_cast<const Tt *>(init), static_cast<Tt *>(out), B, T, 1, T, 1};
        if (algo == LPC_ALGO_CHUNKED) {
            if (workspace_bytes < chunked_forward_workspace(sizeof(Tt), B, T, 1, 1))
                return LPC_ERR_WORKSPACE;
            return cuda_status(chunked_forward<Tt>(p, true, workspace, workspace_bytes, s));
        }
        return cuda_status(plain_forward<Tt>(p, true, s));
    };
    return dtype == LPC_F32 ? run(float{}) : run(double{});
}

size_t lpc_b200_scan_backward_workspace_size(int dtype, int algo, int64_t B, int64_t T) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, 1)) return 0;
    if (resolve_algo(algo, B, T, 1, 1) != LPC_ALGO_CHUNKED) return 0;
    return chunked_backward_workspace(dtype == LPC_F32 ? 4 : 8, B, T, 1, 1);
}

int lpc_b200_scan_backward(int dtype, int algo, const void *grad_out, const void *decay,
                           const void *init, const void *out, void *grad_impulse,
                           void *grad_decay, void *grad_init, int64_t B, int64_t T,
                           void *workspace, size_t workspace_bytes, void *stream) {
    if (!dtype_ok(dtype) || !sizes_ok(B, T, 1)) return LPC_ERR_INVALID_ARGUMENT;
    if (B > 0 && T > 0 && (!grad_out || !decay || !out || !grad_impulse))
        return LPC_ERR_INVALID_ARGUMENT;
    if (B == 0) return LPC_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t esz = dtype == LPC_F32 ? 4 : 8;
    if (T == 0) {
        if (grad_init) cudaMemsetAsync(grad_init, 0, (size_t)B * esz, s);
        return cuda_status(cudaGetLastError());
    }
    algo = resolve_algo(algo, B, T, 1, 1);
    auto run = [&](auto tag) -> int {
        using Tt = decltype(tag);
        BwdArgs<Tt> p{static_cast<const Tt *>(grad_out), static_cast<const Tt *>(decay),
                      static_cast<const Tt *>(init), static_cast<const Tt *>(out),
                      static_cast<Tt *>(grad_impulse), static_cast<Tt *>(grad_decay),
                      static_cast<Tt *>(grad_init), B, T, 1, T, 1};
        if (algo == LPC_ALGO_CHUNKED) {
            if (workspace_bytes < chunked_backward_workspace(sizeof(Tt), B, T, 1, 1))
                return LPC_ERR_WORKSPACE;
            return cuda_status(chunked_backward<Tt>(p, true, workspace, workspace_bytes, s));
        }
        return cuda_status(plain_backward<Tt>(p, true, s));
    };
    return dtype == LPC_F32 ? run(float{}) : run(double{});
}

}  // extern "C"
