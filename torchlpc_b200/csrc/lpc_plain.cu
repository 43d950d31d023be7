// Plain sequential all-pole filter: one warp per signal.
//
// Forward  y[t]  = x[t] - sum_i A[t,i] y[t-i-1]           (y[-k-1] = zi[k])
// Backward gx[t] = gy[t] - sum_i A[t+i+1,i] gx[t+i+1]     (gx beyond T is 0)
//          gzi[k] = gx[-1-k] (the same filter run N steps into negative time)
//          gA[t,i] = -gx[t] y[t-i-1]   (time-invariant A: summed over t)
//
// Layout of the work: the warp stages R time steps of coefficients and input
// into shared memory with cp.async (double buffered, coalesced and 16-byte
// vectorised where the alignment allows), lane 0 runs the recurrence with the
// N-tap history in registers (a ring indexed by compile-time positions, so no
// register moves per step), and the warp writes the outputs back coalesced.
// The backward stages the coefficient diagonal A[t+i+1, i] skewed into shared
// memory so that one step's N taps are contiguous (vector loads, no
// per-step gather), and fuses grad_A / grad_zi into the batch epilogue.
//
// Orders above 32 run the warp-split variants at the bottom of this file:
// lane j owns taps i = j mod 32, the history lives in a shared-memory ring and
// every step ends with a warp reduction.
#include "lpc_plain.cuh"

namespace lpcb {

constexpr int kPlainWarps = 2;

template <typename T>
__device__ __forceinline__ bool aligned16(const T *p) {
    return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

// Copy `count` contiguous elements (vector body when the source is aligned,
// element tail).  All 32 lanes call it; `dst` must be 16-byte aligned.
template <typename T>
__device__ __forceinline__ void warp_copy_async(T *dst, const T *src, int count, int lane) {
    constexpr int V = 16 / sizeof(T);
    int done = 0;
    if (aligned16(src)) {
        const int nv = count / V;
        for (int v = lane; v < nv; v += 32) cp_async<16>(dst + v * V, src + v * V);
        done = nv * V;
    }
    for (int e = done + lane; e < count; e += 32) cp_async<sizeof(T)>(dst + e, src + e);
}

template <typename T, int NP>
__device__ __forceinline__ T hist_dot(const T *a, const T (&h)[NP], int u_minus_1, T acc) {
    // acc - sum_i a[i] * h[(u-1-i) mod NP].  The older taps go into four
    // independent partial sums (short chains that overlap the previous step)
    // and the newest history value enters last, so the loop-carried path of
    // the recurrence is one FMA.
    if constexpr (NP < 4) {
#pragma unroll
        for (int i = NP - 1; i >= 0; --i) acc = fma(-a[i], h[(u_minus_1 - i + 2 * NP) % NP], acc);
        return acc;
    } else {
        T ps[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int i = NP - 1; i >= 1; --i) ps[i & 3] = fma(a[i], h[(u_minus_1 - i + 2 * NP) % NP], ps[i & 3]);
        acc = acc - ((ps[0] + ps[1]) + (ps[2] + ps[3]));
        return fma(-a[0], h[(u_minus_1 + 2 * NP) % NP], acc);
    }
}

template <typename T, int NP, int R>
__device__ __forceinline__ void load_row_vec(T (&dst)[NP], const T *src) {
    if constexpr (sizeof(T) * NP % 16 == 0) {
        constexpr int V = 16 / sizeof(T);
        using V4 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
#pragma unroll
        for (int v = 0; v < NP / V; ++v) {
            V4 q = reinterpret_cast<const V4 *>(src)[v];
            const T *qs = reinterpret_cast<const T *>(&q);
#pragma unroll
            for (int j = 0; j < V; ++j) dst[v * V + j] = qs[j];
        }
    } else {
#pragma unroll
        for (int i = 0; i < NP; ++i) dst[i] = src[i];
    }
}

// ----------------------------------------------------------------------------
// Forward, NP <= 32.
// ----------------------------------------------------------------------------
template <typename T, int NP, bool NEG>
__global__ void __launch_bounds__(32 * kPlainWarps) fwd_plain_kernel(FwdArgs<T> p) {
    constexpr int R = plain_rows(NP);
    constexpr int PER_WARP = 2 * R * NP + 3 * R;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t b = (int64_t)blockIdx.x * kPlainWarps + warp;
    if (b >= p.B) return;
    const int64_t Tn = p.T;
    const int N = (int)p.N;
    T *Abuf = reinterpret_cast<T *>(smem_raw) + warp * PER_WARP;
    T *xbuf = Abuf + 2 * R * NP;
    T *ybuf = xbuf + 2 * R;
    const T *Ab = p.A + b * p.a_stride_b;
    const T *xb = p.x + b * Tn;
    T *yb = p.y + b * Tn;

    if (N < NP)
        for (int e = lane; e < 2 * R * NP; e += 32)
            if (e % NP >= N) Abuf[e] = T(0);

    const int64_t nb = (Tn + R - 1) / R;
    auto load = [&](int64_t k) {
        T *As = Abuf + (k & 1) * R * NP;
        T *xs = xbuf + (k & 1) * R;
        const int64_t t0 = k * R;
        const int rows = (int)min64(R, Tn - t0);
        if (rows < R) {
            for (int e = rows * NP + lane; e < R * NP; e += 32) As[e] = T(0);
            for (int e = rows + lane; e < R; e += 32) xs[e] = T(0);
        }
        if (p.a_stride_t == N && N == NP) {
            warp_copy_async(As, Ab + t0 * N, rows * N, lane);
        } else {
            for (int e = lane; e < rows * N; e += 32) {
                const int r = e / N, i = e - r * N;
                cp_async<sizeof(T)>(As + r * NP + i, Ab + (t0 + r) * p.a_stride_t + i);
            }
        }
        warp_copy_async(xs, xb + t0, rows, lane);
    };

    T h[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        const int i = NP - 1 - j;  // h[NP-1-i] holds y[-1-i]
        h[j] = (p.zi != nullptr && i < N) ? p.zi[b * N + i] : T(0);
    }

    load(0);
    cp_async_commit();
    for (int64_t k = 0; k < nb; ++k) {
        if (k + 1 < nb) load(k + 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncwarp();
        if (lane == 0) {
            const T *As = Abuf + (k & 1) * R * NP;
            const T *xs = xbuf + (k & 1) * R;
            // the next step's coefficient row is read while this step's
            // dot product runs (the shared-memory latency stays off the chain)
            T a[NP];
            load_row_vec<T, NP, R>(a, As);
#pragma unroll 1
            for (int blk = 0; blk < R / NP; ++blk) {
#pragma unroll
                for (int u = 0; u < NP; ++u) {
                    const int r = blk * NP + u;
                    T an[NP] = {};
                    if (r + 1 < R) load_row_vec<T, NP, R>(an, As + (r + 1) * NP);
                    T ac[NP];
#pragma unroll
                    for (int i = 0; i < NP; ++i) ac[i] = NEG ? -a[i] : a[i];
                    const T v = hist_dot<T, NP>(ac, h, u - 1, xs[r]);
                    h[u] = v;
                    ybuf[r] = v;
#pragma unroll
                    for (int i = 0; i < NP; ++i) a[i] = an[i];
                }
            }
        }
        __syncwarp();
        const int64_t t0 = k * R;
        const int rows = (int)min64(R, Tn - t0);
        for (int r = lane; r < rows; r += 32) yb[t0 + r] = ybuf[r];
        __syncwarp();
    }
}

// ----------------------------------------------------------------------------
// Backward, NP <= 32.
// ----------------------------------------------------------------------------
template <typename T, int NP, bool NEG>
__global__ void __launch_bounds__(32 * kPlainWarps) bwd_plain_kernel(BwdArgs<T> p) {
    constexpr int R = plain_rows(NP);
    constexpr int PER_WARP = 2 * R * NP + 3 * R + 2 * (R + NP);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t b = (int64_t)blockIdx.x * kPlainWarps + warp;
    if (b >= p.B) return;
    const int64_t Tn = p.T;
    const int N = (int)p.N;
    T *Dbuf = reinterpret_cast<T *>(smem_raw) + warp * PER_WARP;  // skewed diagonal
    T *gbuf = Dbuf + 2 * R * NP;
    T *gxbuf = gbuf + 2 * R;
    T *ybuf = gxbuf + R;  // 2 stages of the R + NP outputs y the batch's grad_A needs
    const T *Ab = p.A + b * p.a_stride_b;
    const T *gyb = p.gy + b * Tn;
    const T *yb = p.y + b * Tn;
    const T *zib = p.zi ? p.zi + b * N : nullptr;
    const bool ti = (p.a_stride_t == 0);
    const int64_t Text = Tn + (p.gzi ? N : 0);
    const int64_t nb = (Text + R - 1) / R;

    // Step tau (0-based, reversed time) is t = T-1-tau.  Slot s of batch k is
    // tau = k*R + s; its taps are D[s][i] = A[t+1+i, i] = A[T-k*R-s+i, i].
    auto load = [&](int64_t k) {
        T *Ds = Dbuf + (k & 1) * R * NP;
        T *gs = gbuf + (k & 1) * R;
        const int64_t top = Tn - k * R;  // row of (s=0, i=0)
        const int64_t r_lo = max64(0, top - (R - 1));
        const int64_t r_hi = min64(Tn - 1, top + N - 1);
        const bool partial = (top + N - 1 > Tn - 1) || (top < R) || (N < NP);
        if (partial) {
            for (int e = lane; e < R * NP; e += 32) Ds[e] = T(0);
            for (int e = lane; e < R; e += 32) gs[e] = T(0);
            __syncwarp();
        }
        if (r_hi >= r_lo) {
            const int64_t cnt = (r_hi - r_lo + 1) * N;
            for (int64_t e = lane; e < cnt; e += 32) {
                const int64_t r = r_lo + e / N;
                const int i = (int)(e - (r - r_lo) * N);
                const int64_t s = top - r + i;
                if (s >= 0 && s < R) cp_async<sizeof(T)>(Ds + s * NP + i, Ab + r * p.a_stride_t + i);
            }
        }
        // gy for t = top-1-s >= 0, reversed into the slots
        const int64_t t_first = top - 1;  // slot 0
        const int nvalid = (int)max64(0, min64(R, t_first + 1));
        for (int s = lane; s < nvalid; s += 32) cp_async<sizeof(T)>(gs + s, gyb + (t_first - s));
        // y[j] for j = jbase .. jbase+R+NP-1 (zi before the signal), so that
        // the grad_A epilogue reads shared memory instead of waiting on a
        // global load per row
        if (p.gA && !ti) {
            T *ys = ybuf + (k & 1) * (R + NP);
            const int64_t jbase = t_first - R + 1 - NP;
            for (int m = lane; m < R + NP; m += 32) {
                const int64_t j = jbase + m;
                if (j >= 0)
                    cp_async<sizeof(T)>(ys + m, yb + j);
                else
                    ys[m] = (zib && -1 - j < N) ? zib[-1 - j] : T(0);
            }
        }
    };

    T h[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) h[j] = T(0);
    T ga_acc = T(0);  // time-invariant grad for tap i = lane (N <= 32)

    load(0);
    cp_async_commit();
    for (int64_t k = 0; k < nb; ++k) {
        if (k + 1 < nb) load(k + 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncwarp();
        if (lane == 0) {
            const T *Ds = Dbuf + (k & 1) * R * NP;
            const T *gs = gbuf + (k & 1) * R;
            T a[NP];
            load_row_vec<T, NP, R>(a, Ds);
#pragma unroll 1
            for (int blk = 0; blk < R / NP; ++blk) {
#pragma unroll
                for (int u = 0; u < NP; ++u) {
                    const int s = blk * NP + u;
                    T an[NP] = {};
                    if (s + 1 < R) load_row_vec<T, NP, R>(an, Ds + (s + 1) * NP);
                    T ac[NP];
#pragma unroll
                    for (int i = 0; i < NP; ++i) ac[i] = NEG ? -a[i] : a[i];
                    const T v = hist_dot<T, NP>(ac, h, u - 1, gs[s]);
                    h[u] = v;
                    gxbuf[s] = v;
#pragma unroll
                    for (int i = 0; i < NP; ++i) a[i] = an[i];
                }
            }
        }
        __syncwarp();
        // Epilogue for the batch: t runs from t_first down to t_first-R+1.
        const int64_t t_first = Tn - 1 - k * R;
        const int nsteps = (int)min64(R, Text - k * R);
        for (int s = lane; s < nsteps; s += 32) {
            const int64_t t = t_first - s;
            if (t >= 0) p.gx[b * Tn + t] = gxbuf[s];
            else if (p.gzi) p.gzi[b * N + (-1 - t)] = gxbuf[s];
        }
        if (p.gA) {
            const int64_t t_lo = max64(0, t_first - (R - 1));
            const int64_t t_hi = t_first;  // inclusive
            if (t_hi >= t_lo) {
                const T sgn = NEG ? T(1) : T(-1);
                if (!ti) {
                    // a row of N taps per step, lanes along the row (coalesced;
                    // 32-bit indices within the batch, no division per element)
                    const int nrow = (int)(t_hi - t_lo + 1);
                    T *gAb = p.gA + (b * Tn + t_lo) * N;
                    const T *ys = ybuf + (k & 1) * (R + NP);
                    const int64_t jbase = t_first - R + 1 - NP;
                    for (int rr = 0; rr < nrow; ++rr) {
                        const int64_t t = t_lo + rr;
                        const T g = sgn * gxbuf[t_first - t];
                        const T *yr = ys + (int)(t - 1 - jbase);  // y[t-1-i] = yr[-i]
                        for (int i = lane; i < N; i += 32) gAb[rr * N + i] = g * yr[-i];
                    }
                } else if (lane < N) {
                    for (int64_t t = t_lo; t <= t_hi; ++t) {
                        const int64_t j = t - 1 - lane;
                        const T yv = j >= 0 ? yb[j] : (zib ? zib[-1 - j] : T(0));
                        ga_acc = fma(sgn * gxbuf[t_first - t], yv, ga_acc);
                    }
                }
            }
        }
        __syncwarp();
    }
    if (p.gA && ti && lane < N) p.gA[b * N + lane] = ga_acc;
}

// ----------------------------------------------------------------------------
// Warp-split variants for orders above 32 (history in a shared-memory ring).
// ----------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T, bool NEG>
__global__ void __launch_bounds__(32) fwd_wide_kernel(FwdArgs<T> p, int ring) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *hist = reinterpret_cast<T *>(smem_raw);  // hist[(t) & (ring-1)] = y[t]
    const int lane = threadIdx.x;
    const int64_t b = blockIdx.x;
    const int N = (int)p.N;
    const int mask = ring - 1;
    const T *Ab = p.A + b * p.a_stride_b;
    for (int i = lane; i < N; i += 32)  // y[-1-i] = zi[i]
        hist[(-1 - i) & mask] = p.zi ? p.zi[b * N + i] : T(0);
    __syncwarp();
    for (int64_t t = 0; t < p.T; ++t) {
        const T *a = Ab + t * p.a_stride_t;
        T part = T(0);
        for (int i = lane; i < N; i += 32) part = fma(a[i], hist[(int)((t - 1 - i) & mask)], part);
        part = warp_sum(part);
        if (NEG) part = -part;
        if (lane == 0) {
            const T v = p.x[b * p.T + t] - part;
            hist[(int)(t & mask)] = v;
            p.y[b * p.T + t] = v;
        }
        __syncwarp();
    }
}

template <typename T, bool NEG>
__global__ void __launch_bounds__(32) bwd_wide_kernel(BwdArgs<T> p, int ring) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *hist = reinterpret_cast<T *>(smem_raw);  // hist[(t) & (ring-1)] = gx[t]
    const int lane = threadIdx.x;
    const int64_t b = blockIdx.x;
    const int N = (int)p.N;
    const int64_t Tn = p.T;
    const int mask = ring - 1;
    const T *Ab = p.A + b * p.a_stride_b;
    const T *yb = p.y + b * Tn;
    const T *zib = p.zi ? p.zi + b * N : nullptr;
    const bool ti = (p.a_stride_t == 0);
    const T sgn = NEG ? T(1) : T(-1);
    for (int i = lane; i < ring; i += 32) hist[i] = T(0);
    __syncwarp();
    const int64_t t_end = p.gzi ? -N : 0;
    for (int64_t t = Tn - 1; t >= t_end; --t) {
        T part = T(0);
        for (int i = lane; i < N; i += 32) {
            const int64_t r = t + 1 + i;
            if (r >= 0 && r < Tn) part = fma(Ab[r * p.a_stride_t + i], hist[(int)(r & mask)], part);
        }
        part = warp_sum(part);
        if (NEG) part = -part;
        const T g = (t >= 0 ? p.gy[b * Tn + t] : T(0)) - part;
        if (lane == 0) {
            hist[(int)(t & mask)] = g;
            if (t >= 0) p.gx[b * Tn + t] = g;
            else p.gzi[b * N + (-1 - t)] = g;
        }
        if (p.gA && t >= 0 && !ti) {
            for (int i = lane; i < N; i += 32) {
                const int64_t j = t - 1 - i;
                const T yv = j >= 0 ? yb[j] : (zib ? zib[-1 - j] : T(0));
                p.gA[(b * Tn + t) * N + i] = sgn * g * yv;
            }
        }
        __syncwarp();
    }
    if (p.gA && ti) {
        // grad of the shared coefficients: sum over t (second pass over gx, y)
        for (int i = lane; i < N; i += 32) {
            T acc = T(0);
            for (int64_t t = 0; t < Tn; ++t) {
                const int64_t j = t - 1 - i;
                const T yv = j >= 0 ? yb[j] : (zib ? zib[-1 - j] : T(0));
                acc = fma(sgn * p.gx[b * Tn + t], yv, acc);
            }
            p.gA[b * N + i] = acc;
        }
    }
}

// ----------------------------------------------------------------------------
// Launchers.
// ----------------------------------------------------------------------------
static int next_pow2(int v) {
    int r = 1;
    while (r < v) r <<= 1;
    return r;
}

template <typename T, int NP, bool NEG>
static cudaError_t launch_fwd_np(const FwdArgs<T> &p, cudaStream_t st) {
    constexpr int R = plain_rows(NP);
    const size_t smem = (size_t)kPlainWarps * (2 * R * NP + 3 * R) * sizeof(T);
    auto kern = fwd_plain_kernel<T, NP, NEG>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t grid = (p.B + kPlainWarps - 1) / kPlainWarps;
    kern<<<(unsigned)grid, 32 * kPlainWarps, smem, st>>>(p);
    return cudaGetLastError();
}

template <typename T, int NP, bool NEG>
static cudaError_t launch_bwd_np(const BwdArgs<T> &p, cudaStream_t st) {
    constexpr int R = plain_rows(NP);
    const size_t smem = (size_t)kPlainWarps * (2 * R * NP + 3 * R + 2 * (R + NP)) * sizeof(T);
    auto kern = bwd_plain_kernel<T, NP, NEG>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t grid = (p.B + kPlainWarps - 1) / kPlainWarps;
    kern<<<(unsigned)grid, 32 * kPlainWarps, smem, st>>>(p);
    return cudaGetLastError();
}

template <typename T>
cudaError_t plain_forward(const FwdArgs<T> &p, bool neg, cudaStream_t st) {
    if (p.B == 0 || p.T == 0) return cudaSuccess;
    const int NP = padded_order(p.N);
    if (neg) {
        if (NP == 1) return launch_fwd_np<T, 1, true>(p, st);
    } else {
        switch (NP) {
#define LPCB_CASE(n) \
    case n: return launch_fwd_np<T, n, false>(p, st);
            LPCB_FOR_EACH_NP(LPCB_CASE)
#undef LPCB_CASE
            default: break;
        }
    }
    const int ring = next_pow2((int)p.N + 1);
    const size_t smem = (size_t)ring * sizeof(T);
    auto kern = neg ? fwd_wide_kernel<T, true> : fwd_wide_kernel<T, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)p.B, 32, smem, st>>>(p, ring);
    return cudaGetLastError();
}

template <typename T>
cudaError_t plain_backward(const BwdArgs<T> &p, bool neg, cudaStream_t st) {
    if (p.B == 0) return cudaSuccess;
    const int NP = padded_order(p.N);
    if (neg) {
        if (NP == 1) return launch_bwd_np<T, 1, true>(p, st);
    } else {
        switch (NP) {
#define LPCB_CASE(n) \
    case n: return launch_bwd_np<T, n, false>(p, st);
            LPCB_FOR_EACH_NP(LPCB_CASE)
#undef LPCB_CASE
            default: break;
        }
    }
    const int ring = next_pow2((int)p.N + 1);
    const size_t smem = (size_t)ring * sizeof(T);
    auto kern = neg ? bwd_wide_kernel<T, true> : bwd_wide_kernel<T, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)p.B, 32, smem, st>>>(p, ring);
    return cudaGetLastError();
}

template cudaError_t plain_forward<float>(const FwdArgs<float> &, bool, cudaStream_t);
template cudaError_t plain_forward<double>(const FwdArgs<double> &, bool, cudaStream_t);
template cudaError_t plain_backward<float>(const BwdArgs<float> &, bool, cudaStream_t);
template cudaError_t plain_backward<double>(const BwdArgs<double> &, bool, cudaStream_t);

}  // namespace lpcb
