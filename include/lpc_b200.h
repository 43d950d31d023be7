/*
 * lpc_b200 — C ABI of the B200 (sm_100a) time-varying all-pole filter.
 *
 *   y[b,t] = x[b,t] - sum_{i<N} A[b,t,i] * y[b,t-i-1],   y[b,-k-1] = zi[b,k]
 *
 * Plain pointers and sizes only (no torch types).  All pointers are DEVICE
 * pointers on the current CUDA device unless stated otherwise; every entry
 * point is asynchronous on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and returns an lpc_status code.  No entry point allocates memory:
 * callers pass a workspace of at least the size the matching *_workspace_size
 * query returns (0 bytes is valid when that query returns 0).
 *
 * Element type: `dtype` is LPC_F32 (float) or LPC_F64 (double) for every
 * floating-point buffer of a call.
 *
 * Coefficient addressing (strides in elements, the last dimension is unit
 * stride):  A[b,t,i] = A[b*a_stride_b + t*a_stride_t + i].  a_stride_t == 0
 * is a time-invariant filter (a (B,N) tensor broadcast over T, e.g.
 * A[:,None,:].expand(-1,T,-1)); its coefficient gradient is then the (B,N)
 * sum over T.  x, y, grad_y, grad_x are dense (B,T) row-major; zi, grad_zi
 * are dense (B,N).
 */
#ifndef LPC_B200_H
#define LPC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum lpc_status {
    LPC_OK = 0,
    LPC_ERR_INVALID_ARGUMENT = 1, /* bad size, stride, dtype or NULL pointer     */
    LPC_ERR_UNSUPPORTED = 2,      /* valid request this build cannot serve        */
    LPC_ERR_WORKSPACE = 3,        /* workspace missing or smaller than required   */
    LPC_ERR_CUDA = 4,             /* a CUDA runtime call failed (launch, memset)  */
    LPC_ERR_TIMEOUT = 5           /* a bounded device-side wait gave up           */
};

enum lpc_dtype { LPC_F32 = 0, LPC_F64 = 1 };

/* Algorithm selection for the forward/backward passes. */
enum lpc_algo {
    LPC_ALGO_AUTO = 0,    /* choose by (B, T, N) and the coefficient stride         */
    LPC_ALGO_PLAIN = 1,   /* one warp per signal, sequential in time               */
    LPC_ALGO_CHUNKED = 2, /* chunked linear-recurrence scan, parallel in time      */
                          /* (orders above 32 run the plain kernels)             */
    LPC_ALGO_TI = 3       /* time-invariant chunked scan (a_stride_t == 0 only;   */
                          /* otherwise as LPC_ALGO_AUTO)                         */
};

/* Human-readable text for a status code (static storage). */
const char *lpc_b200_status_string(int status);

/* ABI version of this library (major*10000 + minor*100 + patch). */
int lpc_b200_version(void);

/* Target chunk length (samples) of the chunked scan, process-wide: the
 * autotuner's knob (no reference counterpart).  <= 0 restores the default,
 * chosen per call by signal length (128 below 65,536 samples, 256 below 2^19,
 * 512 from there; 1024 for ragged batches), and lpc_b200_chunk_length
 * then returns 0.  Values are clamped to [32, 4096] and rounded up to an even
 * number of the kernel's windows.  Workspace sizes follow the current
 * setting, so change it only between calls. */
int lpc_b200_set_chunk_length(int64_t samples);
int64_t lpc_b200_chunk_length(void);

/* ---------------------------------------------------------------------------
 * Forward filter.
 * Replaces the reference operator torchlpc::lpc(x, A, zi) -> y
 *   (torchlpc/csrc/scan_cpu.cpp:143-164 CPU, torchlpc/csrc/cuda/lpc.cu:115-175
 *    CUDA; schema scan_cpu.cpp:169), called from LPC.forward (core.py:161-163).
 * zi may be NULL (zero initial conditions).  y must not alias x.
 * ------------------------------------------------------------------------- */
size_t lpc_b200_forward_workspace_size(int dtype, int algo, int64_t B, int64_t T,
                                       int64_t N, int64_t a_stride_t);

int lpc_b200_forward(int dtype, int algo, const void *x, const void *A,
                     const void *zi, void *y, int64_t B, int64_t T, int64_t N,
                     int64_t a_stride_b, int64_t a_stride_t, void *workspace,
                     size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------------
 * Fused backward: grad_x, grad_A and grad_zi of the loss given grad_y, in one
 * pass over time (reversed filter with the diagonally shifted coefficients
 * A[t+i+1,i]; grad_A[t,i] = -grad_x[t]*y[t-i-1] fused into the epilogue).
 * Replaces LPC.backward (torchlpc/core.py:186-229).
 * y is the forward output saved for backward.  grad_A is (B,T,N) dense, or
 * (B,N) when a_stride_t == 0.  grad_A and grad_zi may be NULL (not wanted);
 * grad_x is always written.  zi may be NULL (zero initial conditions).
 * ------------------------------------------------------------------------- */
size_t lpc_b200_backward_workspace_size(int dtype, int algo, int64_t B, int64_t T,
                                        int64_t N, int64_t a_stride_t);

int lpc_b200_backward(int dtype, int algo, const void *grad_y, const void *A,
                      const void *zi, const void *y, void *grad_x, void *grad_A,
                      void *grad_zi, int64_t B, int64_t T, int64_t N,
                      int64_t a_stride_b, int64_t a_stride_t, void *workspace,
                      size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------------
 * Boundary-state checkpointing (chunked scan, time-varying coefficients).
 * Replaces what LPC.setup_context saves for the backward
 * (torchlpc/core.py:179-184 keeps (A, zi, y)): the checkpointed forward
 * writes y and, into `states`, the exact N-sample state entering every
 * half-chunk of the scan; the checkpointed backward then needs x and those
 * states instead of y: it recomputes y inside its workspace with one exact
 * pass over independent half-chunks (no maps, no look-back), then runs the
 * fused backward on it.  The gradients are those of lpc_b200_backward.
 * y is therefore not held between the two calls; the backward's workspace
 * holds a B*T copy while it runs.
 * lpc_b200_checkpoint_chunk gives the chunk length the current setting picks
 * for signals of T samples; pass the same chunk_len to both calls (it fixes
 * how the signal is cut, so the chunk-length setting may change in between).
 * lpc_b200_checkpoint_elems gives the number of elements of `states` (dtype
 * as x), about 2*B*T*N/chunk_len.  a_stride_t must be at least N
 * (time-invariant coefficients return LPC_ERR_UNSUPPORTED: their backward
 * runs the time-invariant scan on y); orders above 32 return
 * LPC_ERR_UNSUPPORTED.
 * ------------------------------------------------------------------------- */
int64_t lpc_b200_checkpoint_chunk(int dtype, int64_t T, int64_t N);

int64_t lpc_b200_checkpoint_elems(int dtype, int64_t B, int64_t T, int64_t N,
                                  int64_t chunk_len);

size_t lpc_b200_forward_checkpointed_workspace_size(int dtype, int64_t B, int64_t T,
                                                    int64_t N, int64_t chunk_len);

int lpc_b200_forward_checkpointed(int dtype, const void *x, const void *A,
                                  const void *zi, void *y, void *states, int64_t B,
                                  int64_t T, int64_t N, int64_t a_stride_b,
                                  int64_t a_stride_t, int64_t chunk_len,
                                  void *workspace, size_t workspace_bytes,
                                  void *stream);

size_t lpc_b200_backward_checkpointed_workspace_size(int dtype, int64_t B, int64_t T,
                                                     int64_t N, int64_t chunk_len);

int lpc_b200_backward_checkpointed(int dtype, const void *grad_y, const void *A,
                                   const void *zi, const void *x, const void *states,
                                   void *grad_x, void *grad_A, void *grad_zi,
                                   int64_t B, int64_t T, int64_t N, int64_t a_stride_b,
                                   int64_t a_stride_t, int64_t chunk_len,
                                   void *workspace, size_t workspace_bytes,
                                   void *stream);

/* ---------------------------------------------------------------------------
 * Forward filter with no workspace argument, for callers that cannot allocate
 * device memory (code that must not call an allocator, such as a real-time
 * audio thread or a host callback, or an FFI binding without a memory
 * manager).  No counterpart in the reference: torchlpc always allocates
 * through torch.
 * Runs the chunked kernel with scratch taken from an 8 MiB array compiled
 * into this library (held on every GPU that loads it, until exit).  Returns
 * LPC_ERR_WORKSPACE when the problem needs more scratch than that (roughly
 * 13 to 50 million samples per call at order 16, more for longer signals),
 * LPC_ERR_UNSUPPORTED for orders above 32.  Every call looks up the array's
 * device address in the current context (cudaGetSymbolAddress, no
 * allocation); the first call on a device also loads the module there, so
 * make that first call before any stream capture.  Every call shares the one
 * array: calls whose work overlaps on the GPU (different streams, or several
 * host threads) race and must be serialised by the caller, and changing the
 * chunk length (lpc_b200_set_chunk_length) while a call is being set up is
 * unsupported (a plan that outgrows the array returns LPC_ERR_WORKSPACE).
 * Nothing is allocated or freed.
 * ------------------------------------------------------------------------- */
int lpc_b200_forward_noalloc(int dtype, const void *x, const void *A,
                             const void *zi, void *y, int64_t B, int64_t T,
                             int64_t N, int64_t a_stride_b, int64_t a_stride_t,
                             void *stream);

/* Status word of the last lpc_b200_forward_noalloc call on the current device
 * (the word sits in the library's own scratch array, where
 * lpc_b200_workspace_status cannot reach it): synchronises `stream` and
 * copies the word to *status (host memory).  Nonzero means a bounded wait of
 * that call gave up and its y is invalid; the call itself still returned
 * LPC_OK, since it returns before the kernel runs.  Allocates nothing. */
int lpc_b200_noalloc_status(unsigned *status, void *stream);

/* ---------------------------------------------------------------------------
 * Failure detection.  No reference counterpart (the reference kernels have no
 * bounded waits).  The chunked kernels' waits on other CTAs are bounded; when
 * one gives up it ORs a code into the status word of the call's workspace
 * (1: a predecessor's flag never appeared, 2: inconsistent flags, 8: a ragged
 * signal with a negative length) and the launch completes instead of hanging.
 * lpc_b200_workspace_status reads that word (synchronises `stream`); the
 * word is cleared by the next chunked call that uses the workspace.
 * lpc_b200_selftest_timeout runs a chunked forward whose look-back waits for
 * a flag nothing sets, with the given spin limit (polls of about a
 * microsecond each), and returns LPC_ERR_TIMEOUT with the recorded word in
 * *status when the wait gave up as designed.
 * ------------------------------------------------------------------------- */
int lpc_b200_workspace_status(const void *workspace, unsigned *status, void *stream);

/* Process-wide error word (no reference counterpart): when set, every chunked
 * kernel whose status word ends nonzero ORs it into *word when its CTAs
 * finish, so a caller learns that a call's outputs are invalid without
 * keeping or reading that call's workspace.  `word` must stay valid and
 * device-writable for as long as it is set: mapped pinned host memory
 * (cudaHostAllocMapped; the host then reads it without a CUDA call) or device
 * memory.  The word is only ever OR-ed into; the caller clears it.  NULL
 * turns the reporting off (the default). */
int lpc_b200_set_error_word(unsigned *word);

size_t lpc_b200_selftest_workspace_size(void);

int lpc_b200_selftest_timeout(void *workspace, size_t workspace_bytes,
                              unsigned spin_limit, unsigned *status, void *stream);

/* ---------------------------------------------------------------------------
 * Ragged batches.  No reference counterpart (the reference operators take a
 * dense (B, T) batch; a ragged batch there is padded to the longest signal).
 * nsig signals are concatenated along time: `offsets` is a DEVICE array of
 * nsig+1 non-decreasing int64 sample offsets; signal s is samples
 * [offsets[s], offsets[s+1]) of x, y, grad_y, grad_x and the same rows of A
 * and grad_A (S rows of N, row stride N); zi and grad_zi are (nsig, N), zi
 * may be NULL.  S = offsets[nsig] bounds the workspace.  One persistent launch
 * covers every signal with the chunked scan; orders above 32 return
 * LPC_ERR_UNSUPPORTED.  A negative signal length is treated as empty and
 * recorded in the workspace status word.
 * ------------------------------------------------------------------------- */
size_t lpc_b200_ragged_workspace_size(int dtype, int64_t nsig, int64_t S, int64_t N);

int lpc_b200_forward_ragged(int dtype, const void *x, const void *A,
                            const int64_t *offsets, const void *zi, void *y,
                            int64_t nsig, int64_t S, int64_t N, void *workspace,
                            size_t workspace_bytes, void *stream);

int lpc_b200_backward_ragged(int dtype, const void *grad_y, const void *A,
                             const int64_t *offsets, const void *zi,
                             const void *y, void *grad_x, void *grad_A,
                             void *grad_zi, int64_t nsig, int64_t S, int64_t N,
                             void *workspace, size_t workspace_bytes,
                             void *stream);

/* ---------------------------------------------------------------------------
 * Order-1 recurrence  out[t] = decay[t]*out[t-1] + impulse[t],  out[-1]=init.
 * Replaces the reference operator torchlpc::scan(impulse, decay, init)
 *   (torchlpc/csrc/scan_cpu.cpp:28-78,124-141; linear_recurrence.cu:232-291;
 *    schema scan_cpu.cpp:168), called from Recurrence (recurrence.py:45-84).
 * init may be NULL (zero).
 * ------------------------------------------------------------------------- */
size_t lpc_b200_scan_workspace_size(int dtype, int algo, int64_t B, int64_t T);

int lpc_b200_scan(int dtype, int algo, const void *impulse, const void *decay,
                  const void *init, void *out, int64_t B, int64_t T,
                  void *workspace, size_t workspace_bytes, void *stream);

/* Gradients of the order-1 recurrence (replaces Recurrence.backward,
 * torchlpc/recurrence.py:92-126): grad_impulse[t] = grad_out[t] +
 * decay[t+1]*grad_impulse[t+1]; grad_decay[t] = grad_impulse[t]*out[t-1];
 * grad_init = decay[0]*grad_impulse[0].  grad_decay/grad_init may be NULL. */
size_t lpc_b200_scan_backward_workspace_size(int dtype, int algo, int64_t B, int64_t T);

int lpc_b200_scan_backward(int dtype, int algo, const void *grad_out,
                           const void *decay, const void *init, const void *out,
                           void *grad_impulse, void *grad_decay, void *grad_init,
                           int64_t B, int64_t T, void *workspace,
                           size_t workspace_bytes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* LPC_B200_H */
