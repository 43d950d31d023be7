/*
 * FP64 sequential oracle for the time-varying all-pole (LPC) filter.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that the CUDA kernels
 * of torchlpc_b200 are compared against; it is never part of the product
 * path. Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py load it.
 *
 * Each function restates the algorithm of the reference (DiffAPF/torchlpc)
 * in plain C with double-precision arithmetic:
 *
 *   forward   y[t] = x[t] - sum_{i<N} A[t,i] * y[t-i-1],  y[-k-1] = zi[k]
 *             torchlpc/csrc/scan_cpu.cpp:106-121 (hot loop), :158 (zi is
 *             prepended reversed), torchlpc/__init__.py:102-103 (zf view).
 *   backward  gx[t]  = gy[t] - sum_i A[t+i+1,i] * gx[t+i+1]   (0 beyond T)
 *             gzi[k] = -sum_{i>=k} A[i-k,i] * gx[i-k]
 *             gA[t,i]= -gx[t] * y[t-i-1]
 *             torchlpc/core.py:186-229 (shifted-A reversed filter, grad_zi
 *             from the N padded outputs, grad_A through unfold), README.md
 *             "Derivation of the gradients" (lines 66-130).
 *   time-invariant grad  ga[i] = sum_t gA[t,i]   (README.md:108-130; autograd
 *             expand-backward of tests/test_vmap.py:41).
 *   scan      out[t] = decay[t]*out[t-1] + impulse[t], out[-1] = init
 *             torchlpc/csrc/scan_cpu.cpp:68-77; backward recurrence.py:92-126.
 *
 * Parity of this restatement is pinned against vectors produced by the
 * reference itself (tests/golden/, generated by tests/golden/make_golden.py).
 *
 * Coefficient addressing: A[b,t,i] = A[b*as_b + t*as_t + i]; as_t == 0
 * expresses a time-invariant filter (an expanded (B,N) tensor).
 * Ragged entry points take offsets[B+1] (int64) into concatenated x/y/A
 * rows; signal b covers rows offsets[b] .. offsets[b+1]-1.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static double zi_or_zero(const double *zi, int64_t N, int64_t b, int64_t k) {
    return zi ? zi[b * N + k] : 0.0;
}

/* y at (signal-relative) time s, where s < 0 reads the initial conditions. */
static double ypad(const double *y, const double *zi, int64_t N, int64_t b,
                   int64_t s) {
    return s >= 0 ? y[s] : zi_or_zero(zi, N, b, -s - 1);
}

static void forward_one(int64_t T, int64_t N, const double *x, const double *A,
                        int64_t as_t, const double *zi, int64_t b, double *y) {
    for (int64_t t = 0; t < T; t++) {
        double acc = x[t];
        const double *a = A + t * as_t;
        for (int64_t i = 0; i < N; i++) acc -= a[i] * ypad(y, zi, N, b, t - i - 1);
        y[t] = acc;
    }
}

static void backward_one(int64_t T, int64_t N, const double *gy,
                         const double *A, int64_t as_t, const double *zi,
                         const double *y, int64_t b, double *gx, double *gA,
                         double *ga, double *gzi) {
    for (int64_t t = T - 1; t >= 0; t--) {
        double acc = gy[t];
        for (int64_t i = 0; i < N; i++) {
            int64_t s = t + i + 1;
            if (s < T) acc -= A[s * as_t + i] * gx[s];
        }
        gx[t] = acc;
    }
    if (gzi) {
        for (int64_t k = 0; k < N; k++) {
            double acc = 0.0;
            for (int64_t i = k; i < N; i++) {
                int64_t s = i - k;
                if (s < T) acc -= A[s * as_t + i] * gx[s];
            }
            gzi[b * N + k] = acc;
        }
    }
    if (gA) {
        for (int64_t t = 0; t < T; t++)
            for (int64_t i = 0; i < N; i++)
                gA[t * N + i] = -gx[t] * ypad(y, zi, N, b, t - i - 1);
    }
    if (ga) {
        for (int64_t i = 0; i < N; i++) {
            double acc = 0.0;
            for (int64_t t = 0; t < T; t++) acc -= gx[t] * ypad(y, zi, N, b, t - i - 1);
            ga[b * N + i] = acc;
        }
    }
}

/* Dense batch [B,T]; x, y row-major with row stride T. */
void oracle_lpc_forward(int64_t B, int64_t T, int64_t N, const double *x,
                        const double *A, int64_t as_b, int64_t as_t,
                        const double *zi, double *y) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < B; b++)
        forward_one(T, N, x + b * T, A + b * as_b, as_t, zi, b, y + b * T);
}

/* gA: [B,T,N] dense or NULL; ga: [B,N] (sum over T) or NULL; gzi: [B,N] or NULL. */
void oracle_lpc_backward(int64_t B, int64_t T, int64_t N, const double *gy,
                         const double *A, int64_t as_b, int64_t as_t,
                         const double *zi, const double *y, double *gx,
                         double *gA, double *ga, double *gzi) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < B; b++)
        backward_one(T, N, gy + b * T, A + b * as_b, as_t, zi, y + b * T, b,
                     gx + b * T, gA ? gA + b * T * N : NULL, ga, gzi);
}

/* Ragged: rows of x/y/A concatenated; A has N values per row (time-varying). */
void oracle_lpc_forward_ragged(int64_t B, int64_t N, const int64_t *offsets,
                               const double *x, const double *A,
                               const double *zi, double *y) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < B; b++) {
        int64_t o = offsets[b], T = offsets[b + 1] - offsets[b];
        forward_one(T, N, x + o, A + o * N, N, zi, b, y + o);
    }
}

void oracle_lpc_backward_ragged(int64_t B, int64_t N, const int64_t *offsets,
                                const double *gy, const double *A,
                                const double *zi, const double *y, double *gx,
                                double *gA, double *gzi) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < B; b++) {
        int64_t o = offsets[b], T = offsets[b + 1] - offsets[b];
        backward_one(T, N, gy + o, A + o * N, N, zi, y + o, b, gx + o,
                     gA ? gA + o * N : NULL, NULL, gzi);
    }
}

/* Order-1 recurrence out[t] = decay[t]*out[t-1] + impulse[t]; init may be NULL. */
void oracle_scan_forward(int64_t B, int64_t T, const double *impulse,
                         const double *decay, const double *init, double *out) {
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < B; b++) {
        double h = init ? init[b] : 0.0;
        for (int64_t t = 0; t < T; t++) {
            h = decay[b * T + t] * h + impulse[b * T + t];
            out[b * T + t] = h;
        }
    }
}

/* Gradients of the order-1 recurrence (recurrence.py:92-126):
 *   gi[t] = go[t] + decay[t+1]*gi[t+1]   (reversed filter, decay shifted by one)
 *   gd[t] = gi[t] * out[t-1]  (out[-1] = init)
 *   ginit = decay[0] * gi[0]                                               */
void oracle_scan_backward(int64_t B, int64_t T, const double *grad_out,
                          const double *decay, const double *init,
                          const double *out, double *grad_impulse,
                          double *grad_decay, double *grad_init) {
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < B; b++) {
        const double *d = decay + b * T, *go = grad_out + b * T, *o = out + b * T;
        double *gi = grad_impulse + b * T;
        double h = 0.0;
        for (int64_t t = T - 1; t >= 0; t--) {
            double dn = (t + 1 < T) ? d[t + 1] : 0.0;
            h = go[t] + dn * h;
            gi[t] = h;
        }
        if (grad_decay)
            for (int64_t t = 0; t < T; t++)
                grad_decay[b * T + t] = gi[t] * (t > 0 ? o[t - 1] : (init ? init[b] : 0.0));
        if (grad_init) grad_init[b] = T > 0 ? d[0] * gi[0] : 0.0;
    }
}
